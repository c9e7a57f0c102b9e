// pq_dst_mma.h -- host interface of the tensor-core row DST (pq_dst_mma.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

namespace pq {

// One launch transforms every baroclinic row (modes 1..L-1, rows jlo..jlo+nj-1)
// of x into y (both FP32, the spectral-row layout: row (mode, j) at
// mode * ls + j * pitch, entry k - 1 for wavenumber or node k = 1..N-1).
struct DstMmaArgs {
    const float* x;
    float* y;
    long long ls;  // elements per mode
    int pitch;
    int N;         // transform length + 1 (ii - 1), a power of two >= 64
    int Kp;        // folded K, padded: max(64, N / 2)
    int nj, jlo;   // rows per mode and the first row
    int rows;      // (L - 1) * nj
    int* status;   // the member's status word (ST_MMA_TIMEOUT)
};

bool dst_mma_supported(int N);
int dst_mma_tile_n(int N);
size_t dst_mma_table_bytes(int N);
// The three-term BF16 split of the folded DST matrices ([parity][term][q][m]).
void dst_mma_table(int N, std::vector<unsigned short>& out);
// A TMA descriptor of the device table (128-byte swizzle, 64 x NT boxes).
int dst_mma_tensor_map(CUtensorMap* map, void* table, int N);
cudaError_t launch_dst_mma(const DstMmaArgs& a, const CUtensorMap& map, cudaStream_t st);

}  // namespace pq
