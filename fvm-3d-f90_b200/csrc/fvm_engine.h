// fvm_engine.h — host runtime: blocks, cases, HBM layout, work lists, ghost
// gather lists and the captured CUDA graph of one time step.
//
// One Engine advances any number of cases (each a set of blocks with its own
// scheme configuration) in lockstep: every RK stage is one persistent launch
// per scheme group over the tile work list, followed by the ghost gather; a
// finalize kernel closes the step (residuals, time, next dt). The whole step
// is captured once into a CUDA graph and replayed.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
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
  int64_t n[3] = {1, 1, 1};
  double dr[3] = {1, 1, 1};
  int bc[6] = {0, 0, 0, 0, 0, 0};
  std::vector<HConn> conns;
  // layout (set by plan)
  int64_t px = 0, py = 0, pz = 0, zpad = 0;
  int64_t slab_off = 0;  // element offset of the block's padded box in a slab
  int64_t org = 0;       // element offset of real cell (0,0,0) in a slab
  int64_t sy = 0, sz = 0;
  double* rhs_dev = nullptr;
};

struct HCase {
  fvm_config cfg;
  std::vector<int> blocks;
  int group = -1;
  int tile = -1;        // forced tile (autotuner result), -1 = heuristic
  int zchunk = 0;       // forced z chunk, 0 = heuristic
};

struct Group {
  StageKernelInfo k;
  int prec = 0, dim = 3, recon = 0, flux = 0, tile = 0;
  bool tb = false;
  int task_off = 0, ntasks = 0;
  int grid = 0;
};

class Engine {
 public:
  Engine();
  ~Engine();

  int add_case(const fvm_config& cfg);
  int add_block(int case_id, const int64_t n[3], const double dr[3], int* blk);
  int set_boundary(int blk, int region, int kind);
  int connect(int blk, const int64_t range[3][2], int donor, const int64_t drange[3][2], const int32_t dtype[3]);

  int set_state(int blk, const double* q);
  int get_state(int blk, double* q, int prim);
  int get_rhs(int blk, double* rhs);
  int step(int nsteps);
  int read_case_state(int case_id, DevCaseState* out);

  // Tuning hooks (autotuner): force tile shape / z chunk of a case.
  int set_tuning(int case_id, int tile, int zchunk);
  // Time one stage launch of every group (ms), for the autotuner.
  int time_stage(int reps, float* ms);

  std::string err;
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
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
  int prepare();  // gather ghosts of role A + initial dt, after state uploads
  int profile_step(float* ms, int* kinds, int cap, int* n);

 private:
  int plan();
  int build_graph();
  int enqueue_step(cudaEvent_t* evs, int nev, int* kinds, int* nlaunch);
  void release();
  int resolve(int blk, int64_t x[3], int* out_blk) const;

  bool planned_ = false;
  bool prepared_ = false;
  int nroles_ = 3;
  int max_stages_ = 3;
  int64_t cap_ = 0;
  double* role_[NROLE] = {nullptr, nullptr, nullptr, nullptr};
  double* visc_ = nullptr;
  double* rhs_all_ = nullptr;
  DevBlock* d_blocks_ = nullptr;
  DevCase* d_cases_ = nullptr;
  DevCaseState* d_state_ = nullptr;
  Task* d_tasks_ = nullptr;
  double* d_partials_ = nullptr;
  int64_t* d_pairs_ = nullptr;
  int* d_counters_ = nullptr;
  int ncounters_ = 0;
  unsigned long long* d_casemax_ = nullptr;
  double* d_staging_ = nullptr;
  size_t staging_bytes_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
  std::vector<DevBlock> h_dblocks_;
};

}  // namespace fvm
