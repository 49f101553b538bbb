// xts_tc.cu -- tensor-core (tcgen05) kernels.
#include "xts_internal.cuh"

namespace xts {

int launch_tf32_exposure(const double*, const double*, int, int, const double*, const double*,
                         const double*, int, double*, cudaStream_t) {
    return set_error(XTS_ERR_ARG, "3xTF32 exposure contraction is not built in this library");
}

}  // namespace xts
