// batch_rec.cu -- the instantiations of k_batch_track with the frequency-map record path
// (batch_kernel.cuh), used for serving rounds that hold a frequency-map job.

#include <cuda_runtime.h>

#include "batch.cuh"
#include "batch_kernel.cuh"

namespace bmadgpu {

const void* batch_rec_kernel(int block, int minb, bool full) {
  struct Entry {
    int block, minb;
    const void* fn;
    const void* fn_lean;
  };
#define BG_BATCH_REC(B, M) {B, M, (const void*)k_batch_track<B, M, true, true>, (const void*)k_batch_track<B, M, true, false>}
  static const Entry kRec[] = {
      BG_BATCH_REC(64, 8),  BG_BATCH_REC(64, 12), BG_BATCH_REC(128, 3), BG_BATCH_REC(128, 4),
      BG_BATCH_REC(128, 5), BG_BATCH_REC(128, 6), BG_BATCH_REC(256, 1), BG_BATCH_REC(256, 2),
      BG_BATCH_REC(256, 3), BG_BATCH_REC(512, 1),
  };
#undef BG_BATCH_REC
  for (const Entry& e : kRec)
    if (e.block == block && e.minb == minb) return full ? e.fn : e.fn_lean;
  return nullptr;
}

// This translation unit's copy of the __constant__ multipole tables.
cudaError_t batch_rec_upload_constants() {
  double cm[22][22], cf[22][22];
  build_cmulti_tables(cm, cf);
  cudaError_t e = cudaMemcpyToSymbol(c_cmulti, cm, sizeof(cm));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_cfull, cf, sizeof(cf));
}

}  // namespace bmadgpu
