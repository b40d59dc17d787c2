/* Oracle pin build: data_ptrs with the members of src/cuda/data_ptrs.h:11-31
 * that the Cartesian and log-spherical kernels read. */
#ifndef AP_REF_DATA_PTRS_H_
#define AP_REF_DATA_PTRS_H_
#include "cuda/utils/pitchptr.h"
#include "data/particle_data.h"
namespace Aperture {
struct data_ptrs {
  pitchptr<Scalar> E1, E2, E3, Ebg1, Ebg2, Ebg3, B1, B2, B3, Bbg1, Bbg2, Bbg3;
  pitchptr<Scalar> J1, J2, J3;
  pitchptr<Scalar> divE, divB;
  pitchptr<Scalar> *Rho;
  particle_data particles;
  photon_data photons;
};
}  // namespace Aperture
#endif
