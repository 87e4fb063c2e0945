// fvm_engine.h — host runtime: cases, blocks, the HBM arena, work lists,
// ghost gather lists and the captured CUDA graph of one time step.
//
// One Engine advances any number of independent cases (each a set of blocks
// with its own scheme configuration) in lockstep: every RK stage is one
// persistent launch per scheme group over the tile work list (groups run as
// parallel graph branches), followed by the ghost gather; a finalize kernel
// closes the step (per-case residuals, time, next dt). The step is captured
// once into a CUDA graph and replayed.
//
// State lives in a persistent arena: one slab per (role, variable) whose
// blocks get ranges from a first-fit allocator. Cases can be added and
// removed between steps (the serving loop does this); re-planning rebuilds
// descriptors, tasks and the graph but never moves or clears live state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/fvm3d.h"
#include "fvm_aux.h"
#include "fvm_types.h"

namespace fvm {

struct HConn {
  int64_t range[3][2];
  int donor;
  int64_t drange[3][2];
  int32_t dtype[3];
};

struct HBlock {
  int case_id = 0;
  bool dead = false;
  bool fresh = true;     // region not yet cleared in the arena
  int64_t n[3] = {1, 1, 1};
  double dr[3] = {1, 1, 1};
  int bc[6] = {0, 0, 0, 0, 0, 0};
  std::vector<HConn> conns;
  // layout
  int64_t px = 0, py = 0, pz = 0, zpad = 0;
  int64_t padded = 0;     // elements of the padded box in one variable slab
  int64_t slab_off = -1;  // element offset of the padded box, -1 = unassigned
  int64_t org = 0;        // offset of real cell (0,0,0) inside the padded box
  int64_t sy = 0, sz = 0;
  double* rhs_dev = nullptr;
  // tensor maps of this block ([role][plane box, z box]), encoded for the
  // arena base, slab offset and box shape in tmap_key; re-plans that keep
  // those reuse them instead of encoding again
  std::vector<CUtensorMap> tmaps;
  int64_t tmap_key[4] = {-1, -1, -1, -1};
};

struct HCase {
  fvm_config cfg;
  std::vector<int> blocks;
  bool dead = false;
  bool fresh = true;    // device state (time, residual history) not initialised
  bool dt_stale = true; // state uploaded since the last step: dt is recomputed from it
  int group = -1;
  int tile = -1;        // forced tile (autotuner result), -1 = heuristic
  int zchunk = 0;       // forced z chunk, 0 = chosen by the queue cost model over the case's group
  int tail_split = 1;   // pieces each task of the last, partial queue round is cut into (1 = none)
  // ghost gather pairs of this case, valid while its blocks keep the arena
  // offsets in pairs_key (topology edits clear pairs_valid); pairs_dev_off is
  // where they sit in the engine's device pair array (-1: not there)
  std::vector<int32_t> pairs_cache;
  std::vector<int64_t> pairs_key;
  bool pairs_valid = false;
  int64_t pairs_dev_off = -1;
};

struct Group {
  StageKernelInfo k;
  int prec = 0, dim = 3, recon = 0, flux = 0, tile = 0;
  bool tb = false;
  int task_off = 0, ntasks = 0;
  int grid = 0;
};

// Padded arena elements one block of this shape occupies in one variable slab.
int64_t padded_cells(int idimension, const int64_t n[3]);

class Engine {
 public:
  Engine();
  ~Engine();

  int add_case(const fvm_config& cfg, int* case_id = nullptr);
  int remove_case(int case_id);
  int add_block(int case_id, const int64_t n[3], const double dr[3], int* blk);
  int set_boundary(int blk, int region, int kind);
  int connect(int blk, const int64_t range[3][2], int donor, const int64_t drange[3][2], const int32_t dtype[3]);
  int reserve(int64_t cells);

  int set_state(int blk, const double* q);
  int get_state(int blk, double* q, int prim);
  // several blocks per call: copies on xstream_ overlap the (un)packing
  int set_states(int n, const int* blk, const double* const* q);
  int get_states(int n, const int* blk, double* const* q);
  int get_rhs(int blk, double* rhs);
  int step(int nsteps);
  int read_case_state(int case_id, DevCaseState* out);
  // every case's state in one copy (index = case id; fresh cases hold zeros)
  int read_all_case_states(std::vector<DevCaseState>* out);
  // true once the case's device state exists (read_case_state would succeed)
  bool has_case_state(int case_id) const {
    return live_case(case_id) && d_state_ && case_id < state_cap_ && !cases[case_id].fresh;
  }

  // Test hook of the tensor-copy timeout path (see fvm_test_drop_tensor_copies).
  int set_drop_copies(bool on);
  // Tuning hooks (autotuner): force tile shape / z chunk of a case.
  int set_tuning(int case_id, int tile, int zchunk);
  int set_tail_split(int case_id, int split);
  // Mean device time of `reps` graph-launched steps (ms).
  int time_stage(int reps, float* ms);

  std::string err;
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  // resident CTAs per SM of each stage kernel at its shared-memory size,
  // found once (the attribute and the occupancy query cost a driver call
  // each, on every re-plan otherwise)
  std::vector<std::pair<const void*, int>> occ_cache_;
  std::vector<HCase> cases;
  std::vector<HBlock> blocks;
  std::vector<Group> groups;
  int64_t ntasks_total = 0;
  int64_t npairs = 0;
  int kernel_launches_per_step = 0;

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* where);
  int ensure_planned();
  int prepare();  // gather ghosts of role A + dt of every case, after state uploads
  int profile_step(float* ms, int* kinds, int cap, int* n);
  int live_case(int case_id) const {
    return case_id >= 0 && case_id < (int)cases.size() && !cases[case_id].dead;
  }
  int live_block(int blk) const { return blk >= 0 && blk < (int)blocks.size() && !blocks[blk].dead; }

 private:
  int layout();
  int plan();
  int build_graph();
  int enqueue_step(cudaEvent_t* evs, int nev, int* kinds, int* nlaunch);
  StageArgs stage_args(int g, int m) const;
  void release();      // free everything (destruction)
  void invalidate() {  // topology changed: re-plan before the next use
    planned_ = false;
    prepared_ = false;
    laid_out_ = false;
  }
  int alloc_range(int64_t size, int64_t* off);
  void free_range(int64_t off, int64_t size);
  int grow_arena(int64_t need);
  int resolve(int blk, int64_t x[3], int* out_blk) const;

  bool planned_ = false;
  bool laid_out_ = false;
  bool prepared_ = false;
  int nroles_ = 3;
  int max_stages_ = 3;
  int64_t cap_ = 0;            // elements per variable slab (0 = no arena yet)
  int64_t reserved_ = 0;       // fixed arena size requested by reserve()
  std::vector<std::pair<int64_t, int64_t>> free_;  // (offset, size), sorted
  double* role_[NROLE] = {nullptr, nullptr, nullptr, nullptr};
  double* visc_ = nullptr;
  DevBlock* d_blocks_ = nullptr;
  DevCase* d_cases_ = nullptr;
  int* d_case_blk_ = nullptr;
  DevCaseState* d_state_ = nullptr;
  int state_cap_ = 0;
  Task* d_tasks_ = nullptr;
  double* d_partials_ = nullptr;
  int32_t* d_pairs_ = nullptr;       // (dst, src) cell offsets within a role slab
  int32_t* d_pairs_alt_ = nullptr;   // the next plan's pair array, assembled on the device
  int* d_counters_ = nullptr;
  int ncounters_ = 0;
  // viscous task lists in d_tasks_, index precision * 2 + (3D ? 0 : 1)
  int vlist_off_[6] = {0, 0, 0, 0, 0, 0}, vlist_n_[6] = {0, 0, 0, 0, 0, 0};
  std::vector<CUtensorMap*> d_tmap_;  // per group: [block][role A..ACC][plane, z] (null: no TMA)
  std::vector<size_t> cap_tmap_;      // their capacities in maps (grown, never shrunk)
  int32_t* d_err_ = nullptr;          // kernel error flag (a tensor copy that did not arrive)
  int* d_dtmask_ = nullptr;           // cases whose dt prepare() recomputes
  int dtmask_cap_ = 0;
  bool drop_copies_ = false;          // test hook: tensor copies armed but not issued
  unsigned long long* d_casemax_ = nullptr;
  // element capacities of the descriptor buffers above (grown, never shrunk)
  size_t cap_pairs_alt_ = 0;
  size_t cap_blocks_ = 0, cap_cases_ = 0, cap_case_blk_ = 0, cap_tasks_ = 0, cap_partials_ = 0, cap_pairs_ = 0,
         cap_counters_ = 0, cap_casemax_ = 0;
  double* d_staging_ = nullptr;
  size_t staging_bytes_ = 0;
  double* d_staging2_ = nullptr;      // second staging buffer of set_states / get_states
  size_t staging2_bytes_ = 0;
  cudaStream_t xstream_ = nullptr;    // their host <-> device copies
  cudaEvent_t xev_[5] = {};           // copied[2], used[2], start
  int ensure_xfer();
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
  // kMultiSteps steps in one graph: runs of steps cost one launch per
  // kMultiSteps (what decides the step rate of small cases)
  static constexpr int kMultiSteps = 8;
  cudaGraph_t graphm_ = nullptr;
  cudaGraphExec_t gexecm_ = nullptr;
  void destroy_graphs();
  cudaError_t launch_steps(int nsteps);
  std::vector<cudaStream_t> side_;  // fork streams for parallel group launches
  std::vector<cudaEvent_t> fork_ev_;
  std::vector<DevBlock> h_dblocks_;
};

}  // namespace fvm
