/* Oracle pin build: curandState and curand_uniform come from ls_host_math.h. */
#include "ls_host_math.h"
