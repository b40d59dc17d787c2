// multi_array<Scalar> and the field types of src/core/multi_array.h and
// src/core/fields.h: pitched device arrays (cudaMallocPitch, like the
// reference's cudaMalloc3D storage) with a host copy.
#ifndef APERTURE_DROPIN_MULTI_ARRAY_H_
#define APERTURE_DROPIN_MULTI_ARRAY_H_

#include <cuda_runtime.h>

#include <vector>

#include "ap_common.h"

namespace Aperture {

template <typename T>
class multi_array {
 public:
  multi_array() = default;
  multi_array(int w, int h = 1, int d = 1) { resize(w, h, d); }
  ~multi_array() { release(); }
  multi_array(const multi_array &) = delete;
  multi_array &operator=(const multi_array &) = delete;
  multi_array(multi_array &&o) noexcept { *this = std::move(o); }
  multi_array &operator=(multi_array &&o) noexcept {
    if (this != &o) {
      release();
      dev_ = o.dev_;
      pitch_ = o.pitch_;
      w_ = o.w_, h_ = o.h_, d_ = o.d_;
      host_ = std::move(o.host_);
      o.dev_ = nullptr;
    }
    return *this;
  }

  void resize(int w, int h = 1, int d = 1) {
    release();
    w_ = w, h_ = h, d_ = d;
    // rows padded to 16 bytes at least, as cudaMalloc3D pads them
    cuda_check(cudaMallocPitch(&dev_, &pitch_, sizeof(T) * w, (size_t)h * d), "multi_array");
    host_.assign((size_t)w * h * d, T(0));
    assign_dev(T(0));
  }
  void assign_dev(T v) {
    if (v == T(0)) {
      cuda_check(cudaMemset2D(dev_, pitch_, 0, sizeof(T) * w_, (size_t)h_ * d_), "assign_dev");
    } else {
      for (auto &x : host_) x = v;
      copy_to_device();
    }
  }
  void copy_to_device() {
    cuda_check(cudaMemcpy2D(dev_, pitch_, host_.data(), sizeof(T) * w_, sizeof(T) * w_,
                            (size_t)h_ * d_, cudaMemcpyHostToDevice),
               "copy_to_device");
  }
  void copy_to_host() {
    cuda_check(cudaMemcpy2D(host_.data(), sizeof(T) * w_, dev_, pitch_, sizeof(T) * w_,
                            (size_t)h_ * d_, cudaMemcpyDeviceToHost),
               "copy_to_host");
  }
  T &operator()(int x, int y = 0, int z = 0) { return host_[x + (size_t)w_ * (y + (size_t)h_ * z)]; }
  T *dev_ptr() { return static_cast<T *>(dev_); }
  size_t pitch() const { return pitch_; }
  int width() const { return w_; }
  int height() const { return h_; }
  int depth() const { return d_; }
  ap_array view() { return ap_array{reinterpret_cast<float *>(dev_), pitch_}; }

 private:
  void release() {
    if (dev_) cudaFree(dev_);
    dev_ = nullptr;
  }
  void *dev_ = nullptr;
  size_t pitch_ = 0;
  int w_ = 0, h_ = 0, d_ = 0;
  std::vector<T> host_;
};

// Staggers of the field components (src/core/fields_impl.hpp:84-99): bit i
// set means the component sits on the cell edge in dim i.
enum class FieldType { E, B, Scalar };

template <int N, typename T>
class field {
 public:
  field() = default;
  void resize(const Quadmesh &mesh, FieldType type, unsigned char scalar_stagger = 0b111) {
    mesh_ = mesh;
    for (int i = 0; i < N; ++i) data_[i].resize(mesh.dims[0], mesh.dims[1], mesh.dims[2]);
    const unsigned char e[3] = {0b110, 0b101, 0b011}, b[3] = {0b001, 0b010, 0b100};
    for (int i = 0; i < N; ++i)
      stagger_[i] = type == FieldType::E ? e[i] : type == FieldType::B ? b[i] : scalar_stagger;
  }
  multi_array<T> &data(int n = 0) { return data_[n]; }
  void initialize() {
    for (int i = 0; i < N; ++i) data_[i].assign_dev(T(0));
  }
  // field::initialize(component, f) (src/core/fields.h:114-140): f(x1, x2,
  // x3) sampled at every cell, guards included, at the component's stagger.
  template <typename Func>
  void initialize(int component, const Func &f) {
    auto &a = data_[component];
    for (int k = 0; k < mesh_.dims[2]; ++k) {
      double x3 = mesh_.pos(2, k, (stagger_[component] >> 2) & 1);
      for (int j = 0; j < mesh_.dims[1]; ++j) {
        double x2 = mesh_.pos(1, j, (stagger_[component] >> 1) & 1);
        for (int i = 0; i < mesh_.dims[0]; ++i) {
          double x1 = mesh_.pos(0, i, stagger_[component] & 1);
          a(i, j, k) = (T)f(x1, x2, x3);
        }
      }
    }
    a.copy_to_device();
  }
  template <typename Func>
  void initialize(const Func &f) {
    for (int i = 0; i < N; ++i) initialize(i, f);
  }

 private:
  Quadmesh mesh_{};
  multi_array<T> data_[N];
  unsigned char stagger_[N] = {};
};

template <typename T>
using vector_field = field<3, T>;
template <typename T>
using scalar_field = field<1, T>;

}  // namespace Aperture

#endif
