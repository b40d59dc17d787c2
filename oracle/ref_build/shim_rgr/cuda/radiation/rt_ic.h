/* Oracle pin build, 1D GR radiation: the class the lab's user_rt_init
 * constructs (src/cuda/radiation/rt_ic.h), reduced to no-ops; the pin
 * never calls user_rt_init, and the tables the user functions read come
 * from the oracle's restatement (ref_rad_gr_shim.cpp). */
#ifndef AP_REF_RGR_RT_IC_H_
#define AP_REF_RGR_RT_IC_H_
namespace Aperture {
struct SimParams;
class inverse_compton {
 public:
  explicit inverse_compton(const SimParams &) {}
  template <typename F>
  void init(const F &, Scalar, Scalar, double = 1.0) {}
};
}  // namespace Aperture
#endif
