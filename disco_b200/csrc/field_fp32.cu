// FP32 compensated form of the displacement sum (DISCO_FP32C).
#include <string>

#include "field.cuh"

namespace disco {

int build_table_fp32(const disco_loop*, int, int, double, HostTable&, std::string& err)
{
    err = "DISCO_FP32C is not available in this build";
    return DISCO_EINVAL;
}

int launch_field_fp32(const FieldArgs&, int, int, int, cudaStream_t, std::string& err)
{
    err = "DISCO_FP32C is not available in this build";
    return DISCO_EINVAL;
}

} // namespace disco
