// Tensor-core (tcgen05) triplet contraction.
#include "pb_triplet.cuh"

namespace pb {

int triplet_tc_workspace_size(int64_t, int, int, size_t *bytes) {
    *bytes = 0;
    return fail(PB_ERR_UNSUPPORTED, "tensor-core triplet contraction is not built yet");
}

int launch_triplet_tc(const void *, int, const void *, int, const void *, int, int64_t, const TripletItem *, int, int,
                      double, double *, void *, size_t, cudaStream_t) {
    return fail(PB_ERR_UNSUPPORTED, "tensor-core triplet contraction is not built yet");
}

}  // namespace pb
