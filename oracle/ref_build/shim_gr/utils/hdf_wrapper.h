/* Oracle pin build: the HDF5 file reader Grid_1dGR::compute_coef opens
 * coef.h5 with (src/utils/hdf_wrapper.h), serving the datasets the driver
 * registers in ref_gr_tables instead of reading a file. */
#ifndef AP_REF_GR_HDF_WRAPPER_H_
#define AP_REF_GR_HDF_WRAPPER_H_
#include <map>
#include <string>
#include <vector>
namespace Aperture {
extern std::map<std::string, std::vector<float>> ref_gr_tables;
enum class H5OpenMode { read_only, read_write };
class H5File {
 public:
  H5File(const std::string &, H5OpenMode) {}
  template <typename T>
  std::vector<T> read_vector(const std::string &name) {
    const std::vector<float> &v = ref_gr_tables.at(name);
    return std::vector<T>(v.begin(), v.end());
  }
};
}  // namespace Aperture
#endif
