// builder_parallel.cu -- chunked parallel connectivity builder (placeholder: sequential walk).
#include "builder_internal.cuh"

namespace astrosim {

Status build_parallel(const Sizes& sz, u64 seed, u64 c0, Network& net, cudaStream_t st) {
    return build_sequential(sz, seed, c0, net, st);
}

}  // namespace astrosim
