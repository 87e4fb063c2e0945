// fvm_types.h — device-visible descriptors shared by the host runtime and the
// kernels of the B200 explicit residual-and-update path.
//
// HBM layout. Every state buffer of an engine is one slab per variable:
//   buffer role r (A, B, C, ACC), variable v:  base_r + v * var_stride
// and every block owns a padded box inside each slab:
//   x: 4 pad cells left (keeps real cell 0 on a 32-byte boundary), pitch
//      rounded up to 4 cells; y: 3 ghost rows each side; z: 3 ghost planes
//      each side in 3D, none in 2D (2D planes evolve independently).
// A block descriptor points at its real cell (0,0,0) of variable 0 in each
// role, so cell (i,j,k) of variable v is  q[role][i + j*sy + k*sz + v*vs],
// with ghost cells at negative or >= n indices.
#pragma once
#include <cuda.h>  // CUtensorMap
#include <stdint.h>

namespace fvm {

enum Role { ROLE_A = 0, ROLE_B = 1, ROLE_C = 2, ROLE_ACC = 3, NROLE = 4 };

constexpr int kPadX = 4;   // left x pad (cells)
constexpr int kGhost = 3;  // ghost layers (defs_ghost_cell.f90:42, nGhost_layers = 3)

// ghost_mask bit r (r = region-1, regions of defs_ghost_cell.f90:129-165):
// set when that region's ghost cells are read from storage (filled by the
// gather kernel); clear when they are the zero-order extrapolation of
// update_ghost_cell_sub, which the kernels apply on load by clamping.
struct DevBlock {
  double* q[NROLE];   // real cell (0,0,0), variable 0, per role
  double* rhs;        // optional last-stage rhs, real range (ni,nj,nk,5) Fortran order
  double* visc;       // optional viscous contribution (same padded layout, role-less)
  int64_t vs;         // variable stride (elements)
  int32_t n[3];       // real cells per axis
  int32_t sy, sz;     // element strides of y and z
  int32_t ghost_mask;
  int32_t case_id;
  int32_t task0;      // first task of this block in the engine task list
  int32_t ntask;      // number of tasks of this block
  int32_t pad_;
  double dr[3];
  double inv_dr[3];
};

struct DevCase {
  double gamma, gm1, kappa, entropy_fix, cfl, dt_fixed;
  double mu, prandtl, kq;      // Navier-Stokes: kq = mu*gamma/(Pr*(gamma-1))
  int32_t limiter;
  int32_t compat;              // 0 reference, 1 textbook
  int32_t timestep_set;
  int32_t idim;
  int32_t rk_stages;
  int32_t nblocks;
  int32_t block0;              // first entry of the case in the case-block index list
  int32_t equation;
  int32_t store_rhs;
  int32_t precision;           // fvm_precision of the case
};

// Per-case evolving scalars, written only by the finalize kernel.
struct DevCaseState {
  double dt;          // dt of the next step
  double t;           // physical time
  double dt_last;     // dt of the last completed step
  double res_abs[6];
  double res_abs0[6];
  double res_rel[6];
  long long step;
  int32_t status;     // 0 ok, FVM_ERR_NONFINITE, FVM_ERR_DIVERGED
  int32_t pad_;
};

struct Task {
  int32_t blk, x0, y0, z0, z1, slot;  // slot: index into the partials array
};

// Partials per task: 5 sums of rhs^2 (last stage) + wave-speed max of the
// new state + spare.
constexpr int kPartStride = 8;

struct StageArgs {
  const Task* tasks;
  int32_t ntasks;
  int32_t* counter;            // work-queue head, zeroed before each launch
  const DevBlock* blocks;
  const DevCase* cases;
  const DevCaseState* cstate;
  double* partials;
  int32_t m;                   // RK stage, 1-based
  int32_t rin, rout, rq0, racc;
  int32_t last;                // last stage of the step: residual + wave speed
  // tensor maps of the prefetching 3D kernels, [block][role A..ACC][plane, z]
  // (null for kernels that load with per-thread copies)
  const CUtensorMap* tmap;
  int32_t* err;                // set to 1 when a tensor copy does not arrive
  int32_t drop_copies;         // test of the timeout path: arm the barrier, skip the copy
};

// Programmatic dependent launch. Inside the step graphs the kernels of a time
// step are launched with programmatic stream serialization, so the CTAs of a
// launch are scheduled while the one before it drains. Every kernel of that
// chain calls pdl_wait() before it touches global memory: it returns once the
// preceding kernel has completed and its writes are visible (at once for a
// kernel launched without the attribute). As every kernel of the chain waits,
// the completion of one implies that of all before it. pdl_trigger() lets the
// next launch be scheduled once every CTA of this one has started; it orders
// no memory. Only the short gather and finalize kernels trigger early: a
// launch scheduled behind a long kernel's tail places its CTAs on the few SMs
// free at that moment (up to 8 gather CTAs per SM) and runs unbalanced.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
#endif

}  // namespace fvm
