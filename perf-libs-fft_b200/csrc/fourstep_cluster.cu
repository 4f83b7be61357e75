// Single-pass four-step C2C for n = 256 x 256 on a thread-block cluster.
//
// A cluster of K = 8 CTAs holds one whole transform (512 KB) in its
// distributed shared memory, so the transform costs one HBM read and one
// HBM write instead of the two round trips of the two-pass four-step
// (fourstep.cu).  With x[n2 a + c] (a < n1 rows, c < n2 columns):
//   1. CTA r loads columns c in [32 r, 32 r + 32) (each row's 32 columns are
//      contiguous; the next member's columns load during this member's
//      work), runs the 256-point column FFTs over a in registers;
//   2. output k1 of column c, times W_n^{c k1}, is element c of row k1: it
//      is stored straight into the row tile of CTA k1 / 32 (remote shared
//      memory stores, which do not stall the thread);
//   3. cluster barrier; CTA r runs the row FFTs over c for rows k1 in
//      [32 r, 32 r + 32) and stores X[k1 + n1 k2] (32 consecutive k1 per k2).
// A cluster barrier before step 2 keeps a row tile from being written while
// its owner still transforms the previous member's rows.
// These are the reference's two twiddled Cooley-Tukey levels
// (src/level_ac_t_c2c.cpp:50-85, src/level_ab_t_c2c.cpp:49-80) with the
// intermediate kept on chip.  Clusters walk the batch; every CTA of a
// cluster takes the same members, so all reach every cluster barrier.
#include <cooperative_groups.h>

#include "kernels.h"
#include "pow2_stages.cuh"
#include "ptx.cuh"

namespace cg = cooperative_groups;

namespace plfft_b200 {

constexpr int kClNL = 256;                  // rows = columns = 256
constexpr int kClK = 8;                     // CTAs per cluster
constexpr int kClCols = kClNL / kClK;       // columns (and rows) per CTA
constexpr int kClE = 16;                    // elements per thread
constexpr int kClT = kClNL / kClE;          // threads per 256-point FFT
constexpr int kClGroups = 16;               // FFT thread groups per CTA
constexpr int kClThreads = kClGroups * kClT;  // 256: each group takes 2 columns / rows

__device__ __forceinline__ float2 cl_two_level(const TwoLevel& p, uint32_t e, int lshift) {
  return cmul(__ldg(p.lo + (e & uint32_t(p.l - 1))), __ldg(p.hi + (e >> lshift)));
}

template <int DIR>
__global__ void __launch_bounds__(kClThreads, 1) fourstep_cluster_kernel(const FourStepClusterLaunch L) {
  using P = P2<kClNL, kClE>;
  constexpr int PITCH = (spad_len_c(kClNL) + 1) & ~1;
  extern __shared__ __align__(128) unsigned char smraw[];
  float2* colbufs = reinterpret_cast<float2*>(smraw);  // two column tiles
  float2* rowbuf = colbufs + 2 * kClCols * PITCH;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = int(cluster.block_rank());
  const int64_t cl_id = int64_t(blockIdx.x) / kClK;
  const int64_t ncl = int64_t(gridDim.x) / kClK;
  const int grp0 = threadIdx.x / kClT;  // first column (phase 1) or row (phase 3) of this group
  const int t = threadIdx.x - grp0 * kClT;
  const int lshift = __ffs(L.tw2.l) - 1;
  auto sync = [&]() { __syncwarp(); };
  // columns 32 r .. 32 r + 31 of member b into a column tile (row a holds
  // them contiguously); one cp.async group per member
  auto load_cols = [&](int64_t b, float2* dst) {
    if (b < L.howmany) {
      const float2* x = L.in + b * L.idist;
#pragma unroll 1
      for (int f = threadIdx.x; f < kClCols * kClNL; f += kClThreads) {
        const int a = f / kClCols, c = f - a * kClCols;
        cp_async8(dst + c * PITCH + spad(a), x + (int64_t(kClNL) * a + r * kClCols + c) * L.istride);
      }
    }
    cp_async_commit();
  };

  load_cols(cl_id, colbufs);
  int it = 0;
  for (int64_t b = cl_id; b < L.howmany; b += ncl, ++it) {
    float2* colbuf = colbufs + (it & 1) * kClCols * PITCH;
    // 1. the next member's columns load into the other tile (last read by
    // this CTA's column FFTs of the previous member) while this one runs
    load_cols(b + ncl, colbufs + ((it + 1) & 1) * kClCols * PITCH);
    cp_async_wait_group<1>();
    __syncthreads();
    // every CTA has finished the previous member's rows: their row tiles may
    // be written again
    cluster.sync();
#pragma unroll 1
    for (int grp = grp0; grp < kClCols; grp += kClGroups) {
      float2* mine = colbuf + grp * PITCH;
      float2 v[kClE];
#pragma unroll
      for (int q = 0; q < kClE; ++q) v[q] = mine[spad(t + kClT * q)];
      st_bfly<kClT, kClE, P::radix(0), 1, 0, DIR>(v, t, L.tw);
      Stages<kClNL, kClE, DIR, 1>::run(v, t, mine, L.tw, sync);
      // 2. output k1 of column c (times W_n^{c k1}) is element c of row k1,
      // owned by CTA k1 / 32: pushed there with remote shared-memory stores
      const int c = r * kClCols + grp;
#pragma unroll
      for (int q = 0; q < kClE; ++q) {
        const int k1 = t + kClT * q;
        const float2 val = twmul<DIR>(v[q], cl_two_level(L.tw2, uint32_t(c) * uint32_t(k1), lshift));
        float2* dst = cluster.map_shared_rank(rowbuf, k1 / kClCols);
        dst[(k1 % kClCols) * PITCH + spad(c)] = val;
      }
    }
    cluster.sync();  // every row element has arrived
    // 3. row FFTs, natural-order results back into the row slots
#pragma unroll 1
    for (int grp = grp0; grp < kClCols; grp += kClGroups) {
      float2* mine = rowbuf + grp * PITCH;
      float2 v[kClE];
#pragma unroll
      for (int q = 0; q < kClE; ++q) v[q] = mine[spad(t + kClT * q)];
      st_bfly<kClT, kClE, P::radix(0), 1, 0, DIR>(v, t, L.tw);
      Stages<kClNL, kClE, DIR, 1>::run(v, t, mine, L.tw, sync);
      sync();
#pragma unroll
      for (int q = 0; q < kClE; ++q) mine[spad(t + kClT * q)] = cscale(v[q], L.scale);
    }
    __syncthreads();
    // X[k1 + 256 k2]: 32 consecutive k1 per k2
    float2* y = L.out + b * L.odist;
#pragma unroll 4
    for (int f = threadIdx.x; f < kClCols * kClNL; f += kClThreads) {
      const int k2 = f / kClCols, j = f - k2 * kClCols;
      y[(int64_t(r * kClCols + j) + int64_t(kClNL) * k2) * L.ostride] = rowbuf[j * PITCH + spad(k2)];
    }
    // the next member's first cluster.sync() orders these reads of rowbuf
    // before any CTA writes into it again
  }
  cp_async_wait_all();  // no copy outlives the CTA
}

int fourstep_cluster_smem() { return 3 * kClCols * ((spad_len(kClNL) + 1) & ~1) * int(sizeof(float2)); }

cudaError_t launch_fourstep_cluster(int dir, const FourStepClusterLaunch& L, int max_clusters, cudaStream_t st) {
  auto kern = dir < 0 ? fourstep_cluster_kernel<-1> : fourstep_cluster_kernel<1>;
  const int smem = fourstep_cluster_smem();
  cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
  if (e != cudaSuccess) return e;
  const int64_t ncl = std::max<int64_t>(1, std::min<int64_t>(max_clusters, L.howmany));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(ncl * kClK));
  cfg.blockDim = dim3(kClThreads);
  cfg.dynamicSmemBytes = size_t(smem);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClK;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, kern, L);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// co-resident clusters of this kernel on the current device (0 if none)
int fourstep_cluster_capacity() {
  const int smem = fourstep_cluster_smem();
  if (cudaFuncSetAttribute(fourstep_cluster_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClK);
  cfg.blockDim = dim3(kClThreads);
  cfg.dynamicSmemBytes = size_t(smem);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClK;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fourstep_cluster_kernel<-1>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace plfft_b200
