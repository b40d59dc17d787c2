/* Oracle pin build: the logger calls of Grid_1dGR::compute_coef print
 * nothing on the host. */
#ifndef AP_REF_GR_LOGGER_H_
#define AP_REF_GR_LOGGER_H_
namespace Aperture {
struct Logger {
  template <typename... Args>
  static void print_info(const char *, const Args &...) {}
  template <typename... Args>
  static void print_debug(const char *, const Args &...) {}
};
}  // namespace Aperture
#endif
