// Prismatic matter step (placeholder until the kernels land).
#include "../../include/disco_b200.h"

extern "C" {

int disco_b200_prismatic(const double*, const double*, const double*, int64_t,
                         const disco_slab_loop*, int32_t, const double*,
                         double*, double*, double*, int32_t*, disco_slab_info*,
                         int32_t*, int8_t*, int64_t, disco_copy*, int64_t, int64_t*)
{
    return DISCO_EINVAL;
}

int disco_b200_finalize(const double*, const double*, const double*, const double*,
                        const double*, const double*, int64_t, const disco_copy*, int64_t,
                        const double*, double*, double*, double*, double*, double*, double*)
{
    return DISCO_EINVAL;
}

}
