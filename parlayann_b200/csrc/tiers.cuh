// The tiered search as a reusable launch sequence: sizing of every tier's
// buffers for a plan and batch size, and the enqueue of the tiers on a stream
// with caller-provided buffers (the index's own, or a batch object's).
#pragma once
#include <cuda_runtime.h>
#include "index.cuh"
#include "search.cuh"
#include "search_emu.cuh"

namespace pann {

struct TierSizes {
  // tier 0: shared-memory seen tables, per-warp global spill tables
  uint32_t S = 0, wb = 0, Sg = 0;
  int wpb = 0, blocks = 0;
  int minb = 3;      // resident blocks the first tier's registers are fitted to (3 or 4)
  bool cta = false;  // every query on one block of the exact-emulation kernel instead of the first tiers
  size_t slots = 0, spill_bytes = 0;
  // hand-off from tier 0 to the emulation tier
  uint32_t logcap = 0, viscap = 0;
  ResumeLayout ly{};
  uint64_t rec_cap = 0;
  size_t handoff_bytes = 0;
  // tier 2: one global seen table per warp
  uint32_t S2 = 0, wb2 = 0;
  int t2_slots = 0;
  size_t t2_bytes = 0;
  // emulation tiers
  uint32_t bits0 = 0, vs = 0, base = 0;
  uint64_t S0 = 0, capA = 0, capB = 0;
  bool emu_smem = false;
  size_t emu_smem_need = 0;
  int e2_slots = 0;
  size_t e2_bytes = 0;
};

struct TierBufs {
  uint32_t* cnt = nullptr;  // >= 16 words; the first 16 are cleared by every enqueue
  uint32_t *redo0 = nullptr, *redo1 = nullptr, *emu = nullptr, *ovf = nullptr, *emu_rec = nullptr,
           *ovf_rec = nullptr;  // nq words each
  uint32_t* gspill = nullptr;   // optional (spill_bytes)
  uint32_t* handoff = nullptr;  // optional (handoff_bytes)
  uint32_t* gt2 = nullptr;      // t2_bytes
  uint32_t* ge2 = nullptr;      // e2_bytes
  const uint32_t* job_list0 = nullptr;  // optional tier-0 job order
  const uint32_t* njobs0 = nullptr;     // optional tier-0 job count in device memory
};

cudaError_t launch_search(int dtype, int metric, bool global_table, const SearchArgs& a, int blocks, int threads,
                          size_t smem, cudaStream_t st, int prec, int minb = 3);
cudaError_t launch_emulate(int dtype, int metric, bool smem_tables, const SearchArgs& a, const EmuArgs& e,
                           int blocks, size_t smem, cudaStream_t st);
// Warps per block of the shared-memory emulation tier (one query per block).
constexpr int EMU_BLOCK_WARPS = 4;
cudaError_t launch_emulate_block(int dtype, int metric, const SearchArgs& a, const EmuArgs& e, int blocks, size_t smem,
                                 cudaStream_t st);
int search_occupancy(int dtype, int metric, bool g, int threads, size_t smem, int minb = 3);
uint32_t tier0_slots(const SearchPlan& p, uint32_t R);

// S_force / wpb_force (0 = automatic) override the tier-0 seen-table slots and
// warps per block.
int size_tiers(const pann_index* idx, const SearchPlan& plan, uint64_t nq, int precision, uint32_t S_force,
               int wpb_force, TierSizes* z, int minb_force = 0);
// side (optional): the index's side stream; the exact-emulation tier then
// also runs a pass beside tier 0's tail on it (idx->ev_fork / ev_join order
// it), taking hand-offs as they are published without waiting for any.
int enqueue_tiers(const pann_index* idx, const SearchPlan& plan, const SearchArgs& a, const TierSizes& z,
                  const TierBufs& b, cudaStream_t st, int precision, uint32_t rerank, cudaStream_t side = nullptr);
// The tier-0 job order farthest-from-the-start-point first (order.cu):
// *order points into idx->order, valid until the next call.
int order_far_first(pann_index* idx, const uint8_t* d_queries, const uint32_t* d_self_ids, const uint32_t* d_starts,
                    uint32_t nq, cudaStream_t st, const uint32_t** order);
// A batch's job order (order.cu): longest beam first, then farthest from the
// first start point, for the nq queries in device memory (read at run time).
size_t batch_order_scratch_bytes(uint32_t max_q);
int order_batch(const pann_index* idx, const uint8_t* d_queries, const uint32_t* d_starts, const uint32_t* d_qL,
                const uint32_t* d_nq, uint32_t max_q, void* scratch, size_t scratch_bytes, uint32_t* d_order,
                cudaStream_t st);
// The multi-parent tile search of the precision form (tile.cu).
// tile_rows > 0 fixes the rows staged per round (CUDA-core scoring), else chosen for occupancy.
int enqueue_tile(const pann_index* idx, const SearchPlan& plan, SearchArgs a, uint32_t parents, uint32_t* job_counter,
                 int precision, uint32_t rerank, cudaStream_t st, uint32_t scorer = 0, uint32_t tile_rows = 0);
// Validates the start points and copies them to idx->starts (cached).
int stage_starts(pann_index* idx, const uint32_t* starts, uint32_t n_start, cudaStream_t st);
// The index's own tier buffers for nq queries (grown as needed).
int index_tier_buffers(pann_index* idx, const TierSizes& z, uint32_t nq, int precision, TierBufs* b);
SearchArgs base_args(const pann_index* idx, const SearchPlan& plan, const uint8_t* d_queries,
                     const uint32_t* d_self_ids, uint32_t nq, const uint32_t* d_starts, uint32_t* d_ids,
                     float* d_dists, uint32_t* d_vis, uint32_t* d_cmps, uint32_t* d_status, uint64_t* d_vis_keys,
                     uint32_t vis_cap);

}  // namespace pann
