// Defines the query stream that the reference's kernel sources declare
// (native/cuda/common.h: `extern cudaStream_t g_query_stream;`, normally
// defined in encode_kernel.cu).  Null selects the per-thread default stream
// (the reference builds with --default-stream per-thread).  Test infrastructure.
#include <cuda_runtime.h>
cudaStream_t g_query_stream = nullptr;
