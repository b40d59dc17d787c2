/* Oracle pin build: SoA records with the members of
 * src/data/particle_data.h:50-76 (the reference generates them with Boost.PP,
 * which is not installed). */
#ifndef AP_REF_PARTICLE_DATA_H_
#define AP_REF_PARTICLE_DATA_H_
#include <cstdint>
#include "core/typedefs.h"
struct particle_data {
  Aperture::Pos_t *x1, *x2, *x3;
  Aperture::Scalar *p1, *p2, *p3, *E, *weight;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
};
struct photon_data {
  Aperture::Pos_t *x1, *x2, *x3;
  Aperture::Scalar *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
};
#endif
