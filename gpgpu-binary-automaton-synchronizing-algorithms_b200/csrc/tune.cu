// tune.cu -- kernel-shape autotuner (placeholder: keeps the defaults).
#include "runtime.cuh"

namespace sbfs {

cudaError_t plan_autotune(sbfs_handle *h, Plan &plan)
{
    (void)h;
    (void)plan;
    return cudaSuccess;
}

}  // namespace sbfs
