// ens_persist.cuh -- the ensemble's persistent kernel (MEU_ENS_PERSISTENT): every
// fused Landau step of every member, whatever its grid size, as work items of ONE
// launch per run of steps.
//
// A work item is one block's share of one pass of one member's step: a column tile
// of Z1 or Z2, a plane of PB, PI or PC, or the member's end-of-step reduction (END).
// The items of one step are listed once on the host (pk_plan), pass-major: all
// members' Z1 tiles (largest grids first), then all PB planes, Z2 tiles, PI planes,
// PC planes and END items; step s of a launch repeats the list.  Every block of the
// persistent grid claims items in list order from one counter and runs them:
//
//   * a member's passes are ordered by one counter per member, done[m], raised by one
//     per finished item.  An item of pass p may start once done[m] counts every item
//     of the member's earlier passes (pk_plan's `need`, plus s * per_step), so the
//     members run ahead of one another and no grid-wide barrier exists;
//   * items are claimed in list order and every item waits only on items listed
//     before it, which running blocks have already claimed: the smallest unfinished
//     item never waits, so the launch cannot deadlock whatever number of blocks is
//     resident (no cooperative launch is needed);
//   * every wait is bounded: one that runs out records MEU_ERR_TIMEOUT in the
//     member's error word and sets the launch's abort flag, after which every block
//     stops claiming and leaves.
//
// One schedule per precision for every size (radix plan 2, 256-thread planes, wide
// column tiles), one order parameter per member.  The items run the same device
// functions as the per-bucket kernels (landau_fused_kernels.cuh), so a member's
// fields and diagnostics equal those of a single handle on that schedule bit for bit.
#pragma once
#include <cstdint>
#include <vector>

#include "landau_fused.cuh"

namespace meu {

constexpr int PK_PV = 2, PK_NTP = 256, PK_V = 1;
constexpr int PK_MAX_STEPS = 64;  // steps per persistent launch

enum PkKind : int { PK_Z1 = 0, PK_PB = 1, PK_Z2 = 2, PK_PI = 3, PK_PC = 4, PK_END = 5 };

// item word: member (17 bits) | kind (3 bits) << 17 | index (12 bits) << 20
__host__ __device__ inline uint32_t pk_item(int m, int kind, int idx) {
  return (uint32_t)m | ((uint32_t)kind << 17) | ((uint32_t)idx << 20);
}
constexpr int PK_MAX_MEMBERS = 1 << 17;

struct PkMember {
  int N;
  int per_step;  // items of the member in one step
  NbList nb;     // block partials of each quantity its END reduces
};

struct PkPlan {
  std::vector<uint32_t> items;  // one step, in claim order
  std::vector<int> need;        // done[m] needed before each item (within its step)
  std::vector<PkMember> mt;     // per member
};

// column tile of the persistent kernel (complex columns per Z1/Z2 item)
template <typename R>
constexpr int pk_tm() {
  return sizeof(R) == 4 ? 16 : 8;
}

// the work list of one step for members of grid sizes N[m] (energy[m]: fort.98 energies on)
PkPlan pk_plan(const std::vector<int>& N, const std::vector<int>& energy, bool f64);

// dynamic shared memory the persistent kernel needs (the largest item of any size)
template <typename R>
size_t pk_smem();

// One launch running nsteps steps of every member.  dCtrl: 2 + members ints, zeroed
// here on st before the launch.  Returns the blocks launched.
template <typename R>
int pk_launch(const LanFusedArgs<R>* dA, const PkMember* dMt, const uint32_t* dItems, const int* dNeed, int L,
              int nsteps, int members, int* dCtrl, cudaStream_t st);

}  // namespace meu
