/* Oracle pin build: curandState and curand_uniform come from rgr_host_math.h. */
#include "rgr_host_math.h"
