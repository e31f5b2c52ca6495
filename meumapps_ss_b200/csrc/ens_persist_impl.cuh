// ens_persist_impl.cuh -- the persistent ensemble kernel of ens_persist.cuh,
// instantiated per precision by ens_persist_f32.cu and ens_persist_f64.cu.
#pragma once
#include "ens_persist.cuh"
#include "landau_fused_kernels.cuh"

namespace meu {
namespace pk {

// polls of a dependency wait before the launch gives up; a poll is one L2 load and a
// 64 ns sleep, so a wait that runs out takes about a second, far above any item
constexpr int WAIT_POLLS = 1 << 21;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// wait until *done >= target: 1 when it is, 0 when the wait runs out, -1 when another
// block aborted the launch
__device__ __forceinline__ int wait_done(const int* done, int target, const int* abort_flag) {
  for (int i = 0; i < WAIT_POLLS; ++i) {
    if (ld_acquire(done) >= target) {
      // the data of the items waited for were written through the generic proxy; the
      // bulk copies (TMA engine) this block issues next read them through the async proxy
      asm volatile("fence.proxy.async.global;\n" ::: "memory");
      return 1;
    }
    if (*(volatile const int*)abort_flag) return -1;
    __nanosleep(64);
  }
  return 0;
}

template <typename R, int N>
constexpr size_t item_smem() {
  using P = fz::Plane<R, N, PK_NTP, PK_PV>;
  constexpr int TM = pk_tm<R>();
  constexpr size_t s1 = lf::z1_smem_base<R, N, PK_V, TM>() +
                        (lf::z1_prefetch<R, N, PK_V, TM>() ? lf::z1_smem_stage<R, N, PK_V, TM>() : 0);
  constexpr size_t s2 = lf::z2_smem<R, N, PK_V, TM>();
  constexpr size_t sp = P::smem_bytes();
  return s1 > s2 ? (s1 > sp ? s1 : sp) : (s2 > sp ? s2 : sp);
}
template <typename R>
constexpr size_t smem_all() {
  constexpr size_t a = item_smem<R, 32>(), b = item_smem<R, 48>(), c = item_smem<R, 64>(), d = item_smem<R, 96>(),
                   e = item_smem<R, 128>();
  size_t m = a;
  m = b > m ? b : m;
  m = c > m ? c : m;
  m = d > m ? d : m;
  m = e > m ? e : m;
  return m;
}
// resident blocks per SM the kernel is compiled for: what the largest item's shared
// memory allows (with 6 KB for the items' static arrays and the runtime reserve), at most 4
template <typename R>
constexpr int min_blocks() {
  constexpr int b = (int)(lf::SM_SMEM / (smem_all<R>() + lf::BLOCK_RESERVED + 6 * 1024));
  return b < 1 ? 1 : (b > 4 ? 4 : b);
}

// One item; a call (not inlined), so that each item kind and size gets its own
// register allocation within the kernel's bound instead of one allocation for the
// union of all of them
template <typename R, int N, int KIND>
__device__ __noinline__ void item_fn(const LanFusedArgs<R>& a, const NbList& nb, int idx) {
  constexpr int TM = pk_tm<R>();
  if constexpr (KIND == PK_Z1) lf::lf_z1_body<R, N, PK_V, PK_PV, TM>(a, idx);
  else if constexpr (KIND == PK_PB) lf::lf_pb_body<R, N, PK_V, PK_PV, PK_NTP, true>(a, 0, idx);
  else if constexpr (KIND == PK_Z2) lf::lf_z2_body<R, N, PK_V, PK_PV, TM>(a, idx);
  else if constexpr (KIND == PK_PI) lf::lf_pi_body<R, N, PK_PV, PK_NTP>(a, PK_V, idx, 0);
  else if constexpr (KIND == PK_PC) lf::lf_pc_body<R, N, PK_PV, PK_NTP>(a, PK_V, idx);
  else lf::lf_step_reduce<PK_NTP>(a, nb);
}
template <typename R, int N>
__device__ __forceinline__ void run_item(const LanFusedArgs<R>& a, const NbList& nb, int kind, int idx) {
  switch (kind) {
    case PK_Z1: item_fn<R, N, PK_Z1>(a, nb, idx); break;
    case PK_PB: item_fn<R, N, PK_PB>(a, nb, idx); break;
    case PK_Z2: item_fn<R, N, PK_Z2>(a, nb, idx); break;
    case PK_PI: item_fn<R, N, PK_PI>(a, nb, idx); break;
    case PK_PC: item_fn<R, N, PK_PC>(a, nb, idx); break;
    default: item_fn<R, N, PK_END>(a, nb, idx); break;
  }
}

// ctrl[0]: claim counter, ctrl[1]: abort flag, ctrl[2 + m]: items of member m finished
template <typename R>
__global__ void __launch_bounds__(PK_NTP, min_blocks<R>())
    k_ens_persist(const LanFusedArgs<R>* __restrict__ A, const PkMember* __restrict__ mt,
                  const uint32_t* __restrict__ items, const int* __restrict__ need, int L, int nsteps, int* ctrl) {
  int* claim = ctrl;
  int* abort_flag = ctrl + 1;
  int* done = ctrl + 2;
  const int total = L * nsteps;
  __shared__ int s_item;
  // thread 0 claims the block's next item while the block runs the current one, so the
  // claim's round trip overlaps work (claims stay in list order per block).  It also keeps
  // the last count it acquired and its member: a later item of that member needing no
  // more is ordered after the finished items by that acquire already, so it starts
  // without another round trip.
  int next = 0, seen_m = -1, seen_v = 0;
  if (threadIdx.x == 0) next = atomicAdd(claim, 1);
  for (;;) {
    if (threadIdx.x == 0) {
      const int g = next;
      int it = -1;
      if (g < total && !*(volatile const int*)abort_flag) {
        const int s = g / L, i = g - s * L;
        const int m = (int)(items[i] & (PK_MAX_MEMBERS - 1));
        const int target = s * mt[m].per_step + need[i];
        const int w = (m == seen_m && target <= seen_v) ? 1 : wait_done(done + m, target, abort_flag);
        if (w == 1) {
          it = g;
          if (m != seen_m || target > seen_v) {
            seen_m = m;
            seen_v = target;
          }
        } else if (w == 0) {
          atomicMax(A[m].err, MEU_ERR_TIMEOUT);
          atomicExch(abort_flag, 1);
        }
      }
      s_item = it;
      if (it >= 0) next = atomicAdd(claim, 1);
    }
    __syncthreads();
    const int g = s_item;
    if (g < 0) break;
    const uint32_t w = items[g % L];
    const int m = (int)(w & (PK_MAX_MEMBERS - 1)), kind = (int)((w >> 17) & 7u), idx = (int)(w >> 20);
    const LanFusedArgs<R>& a = A[m];  // fields read where the item uses them
    switch (mt[m].N) {
      case 32: run_item<R, 32>(a, mt[m].nb, kind, idx); break;
      case 48: run_item<R, 48>(a, mt[m].nb, kind, idx); break;
      case 64: run_item<R, 64>(a, mt[m].nb, kind, idx); break;
      case 96: run_item<R, 96>(a, mt[m].nb, kind, idx); break;
      default: run_item<R, 128>(a, mt[m].nb, kind, idx); break;
    }
    // every thread's writes of the item (the barrier), then one release of the member's
    // counter (cumulative: it orders the block's writes before the count)
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;\n" ::"l"(done + m) : "memory");
  }
}

}  // namespace pk

template <typename R>
size_t pk_smem() {
  return pk::smem_all<R>();
}

template <typename R>
int pk_launch(const LanFusedArgs<R>* dA, const PkMember* dMt, const uint32_t* dItems, const int* dNeed, int L,
              int nsteps, int members, int* dCtrl, cudaStream_t st) {
  if (L < 1 || nsteps < 1 || (int64_t)L * nsteps >= ((int64_t)1 << 30))
    throw CudaError("persistent ensemble: work list out of range", MEU_ERR_BADARG);
  auto k = pk::k_ens_persist<R>;
  const size_t smem = pk_smem<R>();
  lf::ensure_smem(k, smem);
  int dev = 0, sms = 0, per = 0;
  MEU_CUDA(cudaGetDevice(&dev));
  MEU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MEU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, PK_NTP, smem));
  if (per < 1) throw CudaError("persistent ensemble kernel does not fit an SM", MEU_ERR_UNSUPPORTED);
  MEU_CUDA(cudaMemsetAsync(dCtrl, 0, sizeof(int) * (2 + (size_t)members), st));
  k<<<per * sms, PK_NTP, smem, st>>>(dA, dMt, dItems, dNeed, L, nsteps, dCtrl);
  MEU_CHECK_LAUNCH();
  return per * sms;
}

}  // namespace meu

#define MEU_PK_INSTANTIATE(R)                                                                                       \
  template size_t meu::pk_smem<R>();                                                                                \
  template int meu::pk_launch<R>(const meu::LanFusedArgs<R>*, const meu::PkMember*, const uint32_t*, const int*, int, \
                                 int, int, int*, cudaStream_t);
