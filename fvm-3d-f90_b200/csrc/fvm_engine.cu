// fvm_engine.cu — host runtime of the B200 residual-and-update path and the
// C ABI of include/fvm3d.h.
//
// The runtime owns device memory only; every entry point validates its
// arguments on the host first (mirroring the reference's mpi%stop("Invalid
// ...") checks, class_space_discret.f90:94-106, class_time_discret.f90:82-108)
// and reports failures as status codes plus a message (ClassError's flag+info,
// global_error.f90:18-33). No CUDA call is made before the first state upload
// or step, so configuration errors surface without a GPU.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fvm_engine.h"

#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

namespace fvm {

namespace {
inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled encode_fn() {
  static PFN_cuTensorMapEncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
  }
  return fn;
}

// Split nz planes into chunks of at most L planes, all of nearly equal length
// (lengths differ by at most one plane).
inline void equal_chunks(int64_t nz, int64_t L, std::vector<int64_t>& z0s) {
  z0s.clear();
  const int64_t nc = std::max<int64_t>(1, (nz + L - 1) / L);
  const int64_t base = nz / nc, extra = nz % nc;
  int64_t z = 0;
  for (int64_t c = 0; c < nc; ++c) {
    z0s.push_back(z);
    z += base + (c < extra ? 1 : 0);
  }
  z0s.push_back(nz);
}

// Makespan of the persistent work queue for tasks of the given costs on
// `slots` CTAs: tasks are taken longest first, each by the CTA that frees
// first (what the atomic task counter does when costs are uniform per plane).
double queue_makespan(std::vector<double>& cost, int slots) {
  std::sort(cost.begin(), cost.end(), std::greater<double>());
  std::vector<double> heap(std::max(1, slots), 0.0);  // min-heap of finish times
  auto cmp = std::greater<double>();
  for (double c : cost) {
    std::pop_heap(heap.begin(), heap.end(), cmp);
    heap.back() += c;
    std::push_heap(heap.begin(), heap.end(), cmp);
  }
  return *std::max_element(heap.begin(), heap.end());
}
inline int stage_roles(int S, int m, int* rin, int* rout) {
  // RK3: A->B, (A,B)->C, (A,C)->A. RK4: A->B, B->C, C->B, B->A (q0 = A).
  static const int r3[3][2] = {{ROLE_A, ROLE_B}, {ROLE_B, ROLE_C}, {ROLE_C, ROLE_A}};
  static const int r4[4][2] = {{ROLE_A, ROLE_B}, {ROLE_B, ROLE_C}, {ROLE_C, ROLE_B}, {ROLE_B, ROLE_A}};
  if (S == 3) {
    *rin = r3[m - 1][0];
    *rout = r3[m - 1][1];
  } else {
    *rin = r4[m - 1][0];
    *rout = r4[m - 1][1];
  }
  return 0;
}
}  // namespace

Engine::Engine() {}

Engine::~Engine() {
  release();
  for (auto s : side_) cudaStreamDestroy(s);
  for (auto e : fork_ev_) cudaEventDestroy(e);
  for (auto e : xev_)
    if (e) cudaEventDestroy(e);
  if (xstream_) cudaStreamDestroy(xstream_);
  if (stream) cudaStreamDestroy(stream);
}

void Engine::release() {
  destroy_graphs();
  // roles beyond nroles_ alias role A: free each allocation once
  for (int r = 0; r < NROLE; ++r) {
    bool alias = false;
    for (int q = 0; q < r; ++q) alias |= (role_[q] == role_[r]);
    if (role_[r] && !alias) cudaFree(role_[r]);
  }
  for (auto& r : role_) r = nullptr;
  void* ptrs[] = {visc_,     d_blocks_,   d_cases_,     d_case_blk_, d_state_, d_tasks_,
                  d_partials_, d_pairs_, d_pairs_alt_, d_counters_, d_casemax_,  d_staging_};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  visc_ = nullptr;
  d_blocks_ = nullptr;
  d_cases_ = nullptr;
  d_case_blk_ = nullptr;
  d_state_ = nullptr;
  state_cap_ = 0;
  d_tasks_ = nullptr;
  d_partials_ = nullptr;
  d_pairs_ = nullptr;
  d_pairs_alt_ = nullptr;
  cap_pairs_alt_ = 0;
  d_counters_ = nullptr;
  d_casemax_ = nullptr;
  cap_blocks_ = cap_cases_ = cap_case_blk_ = cap_tasks_ = cap_partials_ = cap_pairs_ = cap_counters_ = cap_casemax_ = 0;
  d_staging_ = nullptr;
  staging_bytes_ = 0;
  if (d_staging2_) cudaFree(d_staging2_);
  d_staging2_ = nullptr;
  staging2_bytes_ = 0;
  for (auto p : d_tmap_)
    if (p) cudaFree(p);
  d_tmap_.clear();
  cap_tmap_.clear();
  if (d_err_) cudaFree(d_err_);
  d_err_ = nullptr;
  if (d_dtmask_) cudaFree(d_dtmask_);
  d_dtmask_ = nullptr;
  dtmask_cap_ = 0;
  for (auto& b : blocks) {
    if (b.rhs_dev) cudaFree(b.rhs_dev);
    b.rhs_dev = nullptr;
    b.slab_off = -1;
    b.fresh = true;
  }
  for (auto& c : cases) c.fresh = true;
  cap_ = 0;
  free_.clear();
  planned_ = false;
  prepared_ = false;
}

int Engine::cuda_fail(cudaError_t e, const char* where) {
  return fail(FVM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

int64_t padded_cells(int idimension, const int64_t n[3]) {
  const int64_t px = round_up(n[0] + kPadX + kGhost, 4);
  const int64_t py = n[1] + 2 * kGhost;
  const int64_t pz = n[2] + 2 * (idimension == 3 ? kGhost : 0);
  return round_up(px * py * pz, 64);
}

// ---------------------------------------------------------------- topology
int Engine::add_case(const fvm_config& c, int* case_id) {
  if (c.struct_size != (int32_t)sizeof(fvm_config)) return fail(FVM_ERR_INVALID, "fvm_config.struct_size mismatch");
  if (c.idimension != 2 && c.idimension != 3) return fail(FVM_ERR_INVALID, "idimension must be 2 or 3");
  if (c.equation != FVM_EQ_EULER && c.equation != FVM_EQ_NAVIER_STOKES)
    return fail(FVM_ERR_INVALID, "Invalid equation type.");
  if (c.reconstruct == FVM_RECON_WCNS)
    return fail(FVM_ERR_UNSUPPORTED, "WCNS has no implementation in the reference");
  if (c.reconstruct != FVM_RECON_SIMPLE && c.reconstruct != FVM_RECON_MUSCL && c.reconstruct != FVM_RECON_WENO)
    return fail(FVM_ERR_INVALID, "Invalid reconstruct scheme.");
  if (c.flux_split == FVM_FLUX_HLLC)
    return fail(FVM_ERR_UNSUPPORTED, "HLLC has no implementation in the reference (its flux stays zero)");
  if (c.flux_split != FVM_FLUX_ROE && c.flux_split != FVM_FLUX_VANLEER && c.flux_split != FVM_FLUX_AUSM)
    return fail(FVM_ERR_INVALID, "Invalid flux split scheme.");
  if (c.limiter != FVM_SCHEME_NULL && (c.limiter < FVM_LIMITER_NONE || c.limiter > FVM_LIMITER_VANALBADA))
    return fail(FVM_ERR_INVALID, "Invalid limiter.");
  if (c.time_scheme >= 102 && c.time_scheme <= 106)
    return fail(FVM_ERR_UNSUPPORTED, "only Runge-Kutta time stepping exists in the reference");
  if (c.time_scheme != FVM_TIME_RUNGE_KUTTA) return fail(FVM_ERR_INVALID, "Invalid time discretization scheme.");
  if (c.rk_stages != 3 && c.rk_stages != 4) return fail(FVM_ERR_INVALID, "rk_stages must be 3 or 4");
  if (c.timestep_set < FVM_DT_FIXED || c.timestep_set > FVM_DT_CFL_LOCAL)
    return fail(FVM_ERR_INVALID, "Invalid timestep type.");
  if (c.timestep_set == FVM_DT_FIXED && c.dt < -1.0E-6) return fail(FVM_ERR_INVALID, "Invalid time step.");
  if (c.timestep_set != FVM_DT_FIXED && !(c.cfl > 0.0)) return fail(FVM_ERR_INVALID, "cfl must be positive");
  if (c.compat != FVM_COMPAT_REFERENCE && c.compat != FVM_COMPAT_TEXTBOOK)
    return fail(FVM_ERR_INVALID, "compat must be 0 or 1");
  if (c.precision < FVM_PREC_FP64_EXACT || c.precision > FVM_PREC_FP32_FLUX)
    return fail(FVM_ERR_INVALID, "precision must be 0, 1 or 2");
  if (!(c.gamma > 1.0)) return fail(FVM_ERR_INVALID, "gamma must exceed 1");
  if (c.equation == FVM_EQ_NAVIER_STOKES && (!(c.mu >= 0.0) || !(c.prandtl > 0.0)))
    return fail(FVM_ERR_INVALID, "Navier-Stokes needs mu >= 0 and prandtl > 0");
  for (const auto& o : cases)
    if (!o.dead && o.cfg.rk_stages != c.rk_stages)
      return fail(FVM_ERR_INVALID, "all cases of one engine share the RK stage count");
  if (cap_ > 0 && nroles_ < (c.rk_stages == 4 ? 4 : 3))
    return fail(FVM_ERR_INVALID, "the arena was laid out for 3 RK stages");
  HCase hc;
  hc.cfg = c;
  // a removed case's slot is taken again (never slot 0, the context's own
  // first case, whose removal fvm_step reports as "no outputs"), so a
  // long-running server's case list, device state array and finalize grid
  // stay the size of its running set
  int slot = -1;
  for (size_t i = 1; i < cases.size() && slot < 0; ++i)
    if (cases[i].dead) slot = (int)i;
  if (slot < 0) {
    cases.push_back(hc);
    slot = (int)cases.size() - 1;
  } else {
    cases[slot] = hc;
  }
  if (case_id) *case_id = slot;
  invalidate();
  return FVM_OK;
}

int Engine::remove_case(int case_id) {
  if (!live_case(case_id)) return fail(FVM_ERR_INVALID, "bad case id");
  HCase& hc = cases[case_id];
  for (int b : hc.blocks) {
    HBlock& B = blocks[b];
    if (B.slab_off >= 0) free_range(B.slab_off, B.padded);
    if (B.rhs_dev) cudaFree(B.rhs_dev);
    B.rhs_dev = nullptr;
    B.slab_off = -1;
    B.dead = true;
    B.conns.clear();
  }
  hc.dead = true;
  invalidate();
  return FVM_OK;
}

int Engine::reserve(int64_t cells) {
  if (cells < 0) return fail(FVM_ERR_INVALID, "negative reservation");
  if (cap_ > 0) return fail(FVM_ERR_STATE, "the arena is already laid out");
  reserved_ = cells;
  return FVM_OK;
}

int Engine::add_block(int case_id, const int64_t n[3], const double dr[3], int* blk) {
  if (!live_case(case_id)) return fail(FVM_ERR_INVALID, "bad case id");
  if (!n || !dr) return fail(FVM_ERR_INVALID, "null nvert / dr");
  for (int d = 0; d < 3; ++d) {
    if (n[d] < 1 || n[d] > (1 << 20)) return fail(FVM_ERR_INVALID, "nvert out of range [1, 2^20]");
    if (!(dr[d] > 0.0) || !std::isfinite(dr[d])) return fail(FVM_ERR_INVALID, "dr must be positive");
  }
  if (padded_cells(cases[case_id].cfg.idimension, n) >= ((int64_t)1 << 31))
    return fail(FVM_ERR_INVALID, "block too large (2^31 padded cells)");
  HBlock b;
  b.case_id = case_id;
  for (int d = 0; d < 3; ++d) {
    b.n[d] = n[d];
    b.dr[d] = dr[d];
  }
  // a removed block's slot is taken again (its arena range was freed)
  int slot = -1;
  for (size_t i = 0; i < blocks.size() && slot < 0; ++i)
    if (blocks[i].dead) slot = (int)i;
  if (slot < 0) {
    blocks.push_back(b);
    slot = (int)blocks.size() - 1;
  } else {
    blocks[slot] = b;
  }
  cases[case_id].blocks.push_back(slot);
  if (blk) *blk = slot;
  invalidate();
  return FVM_OK;
}

int Engine::set_boundary(int blk, int region, int kind) {
  if (!live_block(blk)) return fail(FVM_ERR_INVALID, "bad block id");
  if (region < 1 || region > 6) return fail(FVM_ERR_INVALID, "region must be 1..6");
  HBlock& b = blocks[blk];
  const int ax = (region - 1) / 2;
  const bool hi = (region - 1) % 2 == 1;
  const int idim = cases[b.case_id].cfg.idimension;
  if (ax == 2 && idim == 2 && kind != FVM_BC_TRANSMISSIVE)
    return fail(FVM_ERR_INVALID, "2D blocks have no k ghost regions to connect");
  if (kind != FVM_BC_TRANSMISSIVE && kind != FVM_BC_PERIODIC && kind != FVM_BC_CONNECTED)
    return fail(FVM_ERR_INVALID, "unknown boundary kind");
  if (kind == FVM_BC_PERIODIC && b.n[ax] < kGhost)
    return fail(FVM_ERR_INVALID, "periodic region needs at least 3 cells along its axis");
  std::vector<HConn> keep;
  for (auto& c : b.conns) {
    const bool same = hi ? (c.range[ax][0] >= b.n[ax]) : (c.range[ax][1] < 0);
    if (!same) keep.push_back(c);
  }
  b.conns = keep;
  b.bc[region - 1] = kind;
  if (kind == FVM_BC_PERIODIC) {
    HConn c;
    for (int d = 0; d < 3; ++d) {
      c.range[d][0] = 0;
      c.range[d][1] = b.n[d] - 1;
      c.drange[d][0] = 0;
      c.drange[d][1] = b.n[d] - 1;
      c.dtype[d] = d + 1;
    }
    if (hi) {
      c.range[ax][0] = b.n[ax];
      c.range[ax][1] = b.n[ax] + 2;
      c.drange[ax][0] = 0;
      c.drange[ax][1] = 2;
    } else {
      c.range[ax][0] = -3;
      c.range[ax][1] = -1;
      c.drange[ax][0] = b.n[ax] - 3;
      c.drange[ax][1] = b.n[ax] - 1;
    }
    c.donor = blk;
    b.conns.push_back(c);
  }
  cases[b.case_id].pairs_valid = false;
  invalidate();
  return FVM_OK;
}

int Engine::connect(int blk, const int64_t range[3][2], int donor, const int64_t drange[3][2],
                    const int32_t dtype[3]) {
  if (!live_block(blk) || !live_block(donor)) return fail(FVM_ERR_INVALID, "bad block id");
  if (!range || !drange || !dtype) return fail(FVM_ERR_INVALID, "null range");
  int seen = 0;
  for (int a = 0; a < 3; ++a) {
    const int d = std::abs(dtype[a]);
    if (d < 1 || d > 3) return fail(FVM_ERR_INVALID, "donor_type is not a signed permutation");
    seen |= 1 << (d - 1);
  }
  if (seen != 7) return fail(FVM_ERR_INVALID, "donor_type is not a signed permutation");
  HBlock& b = blocks[blk];
  const HBlock& dn = blocks[donor];
  if (dn.case_id != b.case_id) return fail(FVM_ERR_INVALID, "donor block belongs to another case");
  HConn c;
  c.donor = donor;
  int out_axis = -1;
  for (int a = 0; a < 3; ++a) {
    c.range[a][0] = range[a][0];
    c.range[a][1] = range[a][1];
    c.drange[a][0] = drange[a][0];
    c.drange[a][1] = drange[a][1];
    c.dtype[a] = dtype[a];
    if (c.range[a][1] < c.range[a][0]) return fail(FVM_ERR_INVALID, "empty range");
    const int64_t s = dtype[a] > 0 ? 1 : -1;
    if (c.drange[a][1] - c.drange[a][0] != s * (c.range[a][1] - c.range[a][0]))
      return fail(FVM_ERR_INVALID, "donor range extent does not match");
    const bool out = c.range[a][1] < 0 || c.range[a][0] >= b.n[a];
    const bool in = c.range[a][0] >= 0 && c.range[a][1] < b.n[a];
    if (out) {
      if (out_axis >= 0) return fail(FVM_ERR_INVALID, "range is not a face ghost box");
      out_axis = a;
      if (c.range[a][0] < -kGhost || c.range[a][1] > b.n[a] + kGhost - 1)
        return fail(FVM_ERR_INVALID, "range beyond the 3 ghost layers");
    } else if (!in) {
      return fail(FVM_ERR_INVALID, "range straddles the block boundary");
    }
  }
  if (out_axis < 0) return fail(FVM_ERR_INVALID, "range holds no ghost cells");
  if (out_axis == 2 && cases[b.case_id].cfg.idimension == 2)
    return fail(FVM_ERR_INVALID, "2D blocks have no k ghost regions to connect");
  for (int a = 0; a < 3; ++a) {
    const int da = std::abs(dtype[a]) - 1;
    for (int s = 0; s < 2; ++s)
      if (c.drange[a][s] < 0 || c.drange[a][s] >= dn.n[da])
        return fail(FVM_ERR_INVALID, "donor range outside the donor's real cells");
  }
  const int region = 2 * out_axis + (c.range[out_axis][0] >= b.n[out_axis] ? 2 : 1);
  if (b.bc[region - 1] == FVM_BC_PERIODIC) {
    // replacing the periodic self-connection of this region
    std::vector<HConn> keep;
    const bool hi = region % 2 == 0;
    for (auto& e : b.conns) {
      const bool same = hi ? (e.range[out_axis][0] >= b.n[out_axis]) : (e.range[out_axis][1] < 0);
      if (!same) keep.push_back(e);
    }
    b.conns = keep;
  }
  b.bc[region - 1] = FVM_BC_CONNECTED;
  b.conns.push_back(c);
  cases[b.case_id].pairs_valid = false;
  invalidate();
  return FVM_OK;
}

// Follow ghost rules until x is a real cell: the lowest out-of-range axis
// first; transmissive clamps, connected maps through the connection whose
// box holds x with the other axes clamped into the block.
int Engine::resolve(int blk, int64_t x[3], int* out_blk) const {
  for (int it = 0; it < 4; ++it) {
    const HBlock& b = blocks[blk];
    int a = -1;
    for (int d = 0; d < 3 && a < 0; ++d)
      if (x[d] < 0 || x[d] >= b.n[d]) a = d;
    if (a < 0) {
      *out_blk = blk;
      return 0;
    }
    const bool hi = x[a] >= b.n[a];
    const int region = 2 * a + (hi ? 2 : 1);
    if (b.bc[region - 1] == FVM_BC_TRANSMISSIVE) {
      x[a] = hi ? b.n[a] - 1 : 0;
      continue;
    }
    int64_t xc[3] = {x[0], x[1], x[2]};
    for (int d = 0; d < 3; ++d)
      if (d != a) xc[d] = std::min<int64_t>(std::max<int64_t>(xc[d], 0), b.n[d] - 1);
    const HConn* hit = nullptr;
    for (const auto& c : b.conns) {
      bool in = true;
      for (int d = 0; d < 3; ++d) in = in && xc[d] >= c.range[d][0] && xc[d] <= c.range[d][1];
      if (in) {
        hit = &c;
        break;
      }
    }
    if (!hit) return -1;
    int64_t y[3];
    for (int d = 0; d < 3; ++d) {
      const int dd = std::abs(hit->dtype[d]) - 1;
      const int64_t s = hit->dtype[d] > 0 ? 1 : -1;
      y[dd] = hit->drange[d][0] + s * (x[d] - hit->range[d][0]);
    }
    blk = hit->donor;
    for (int d = 0; d < 3; ++d) x[d] = y[d];
  }
  return -1;
}

// ---------------------------------------------------------------- planning
int Engine::set_drop_copies(bool on) {
  if (drop_copies_ != on) {
    drop_copies_ = on;
    planned_ = false;  // the step graph carries the flag in its kernel arguments
  }
  return FVM_OK;
}

int Engine::set_tuning(int case_id, int tile, int zchunk) {
  if (!live_case(case_id)) return fail(FVM_ERR_INVALID, "bad case id");
  if (tile < -1 || tile >= kNumTiles) return fail(FVM_ERR_INVALID, "bad tile index");
  if (zchunk < 0) return fail(FVM_ERR_INVALID, "bad z chunk");
  if (cases[case_id].tile == tile && cases[case_id].zchunk == zchunk) return FVM_OK;
  cases[case_id].tile = tile;
  cases[case_id].zchunk = zchunk;
  invalidate();  // the arena and every case's state stay where they are
  return FVM_OK;
}

int Engine::set_tail_split(int case_id, int split) {
  if (!live_case(case_id)) return fail(FVM_ERR_INVALID, "bad case id");
  if (split < 1 || split > 8) return fail(FVM_ERR_INVALID, "bad tail split");
  if (cases[case_id].tail_split == split) return FVM_OK;
  cases[case_id].tail_split = split;
  invalidate();
  return FVM_OK;
}

// ---------------------------------------------------------------- arena
int Engine::alloc_range(int64_t size, int64_t* off) {
  for (size_t i = 0; i < free_.size(); ++i) {
    if (free_[i].second >= size) {
      *off = free_[i].first;
      free_[i].first += size;
      free_[i].second -= size;
      if (free_[i].second == 0) free_.erase(free_.begin() + i);
      return 0;
    }
  }
  return -1;
}

void Engine::free_range(int64_t off, int64_t size) {
  free_.push_back({off, size});
  std::sort(free_.begin(), free_.end());
  std::vector<std::pair<int64_t, int64_t>> m;
  for (auto& r : free_) {
    if (!m.empty() && m.back().first + m.back().second == r.first)
      m.back().second += r.second;
    else
      m.push_back(r);
  }
  free_ = m;
}

// Replace the arena by one of at least `need` elements per slab, moving the
// live blocks' boxes (all roles and the viscous slab) to their new offsets.
int Engine::grow_arena(int64_t need) {
  const int64_t ncap = round_up(std::max(need, cap_), 64);
  double* nr[NROLE] = {nullptr, nullptr, nullptr, nullptr};
  for (int r = 0; r < nroles_; ++r) {
    cudaError_t e = cudaMalloc(&nr[r], sizeof(double) * 5 * ncap);
    if (e != cudaSuccess) {
      for (int q = 0; q < r; ++q) cudaFree(nr[q]);
      return fail(FVM_ERR_NOMEM, std::string("state allocation: ") + cudaGetErrorString(e));
    }
    CK(cudaMemsetAsync(nr[r], 0, sizeof(double) * 5 * ncap, stream));
  }
  double* nv = nullptr;
  if (visc_) {
    CK(cudaMalloc(&nv, sizeof(double) * 5 * ncap));
    CK(cudaMemsetAsync(nv, 0, sizeof(double) * 5 * ncap, stream));
  }
  // lay the live, already placed blocks out contiguously in the new arena
  int64_t off = 0;
  for (auto& b : blocks) {
    if (b.dead || b.slab_off < 0) continue;
    for (int r = 0; r < nroles_; ++r)
      for (int v = 0; v < 5; ++v)
        CK(cudaMemcpyAsync(nr[r] + off + v * ncap, role_[r] + b.slab_off + v * cap_, sizeof(double) * b.padded,
                           cudaMemcpyDeviceToDevice, stream));
    b.slab_off = off;
    off += b.padded;
  }
  CK(cudaStreamSynchronize(stream));
  for (int r = 0; r < nroles_; ++r)
    if (role_[r]) cudaFree(role_[r]);
  if (visc_) cudaFree(visc_);
  for (int r = 0; r < NROLE; ++r) role_[r] = (r < nroles_) ? nr[r] : nr[ROLE_A];
  visc_ = nv;
  cap_ = ncap;
  free_.clear();
  if (off < cap_) free_.push_back({off, cap_ - off});
  return FVM_OK;
}

// ---------------------------------------------------------------- planning
int Engine::ensure_planned() {
  if (planned_) return FVM_OK;
  return plan();
}

// Layout of the live blocks in the arena: region coverage checks, padded
// boxes, arena ranges for new blocks (cleared once). Enough for state
// uploads and downloads; plan() adds the work lists and the step graph.
int Engine::layout() {
  std::vector<int> live_cases, live_blocks;
  for (size_t c = 0; c < cases.size(); ++c)
    if (!cases[c].dead) live_cases.push_back((int)c);
  for (size_t b = 0; b < blocks.size(); ++b)
    if (!blocks[b].dead) live_blocks.push_back((int)b);
  if (live_cases.empty()) return fail(FVM_ERR_STATE, "no case configured");
  if (live_blocks.empty()) return fail(FVM_ERR_STATE, "no block added");
  if (!stream) {
    CK(cudaGetDevice(&device));
    CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  }
  max_stages_ = cases[live_cases[0]].cfg.rk_stages;
  bool any_ns = false;
  for (int c : live_cases) any_ns |= cases[c].cfg.equation == FVM_EQ_NAVIER_STOKES;

  // -- coverage of connected regions
  for (int bi : live_blocks) {
    const HBlock& b = blocks[bi];
    for (int region = 1; region <= 6; ++region) {
      if (b.bc[region - 1] == FVM_BC_TRANSMISSIVE) continue;
      const int ax = (region - 1) / 2;
      const bool hi = (region - 1) % 2 == 1;
      const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
      std::vector<char> cov((size_t)3 * b.n[t1] * b.n[t2], 0);
      for (const auto& c : b.conns) {
        const bool same = hi ? (c.range[ax][0] >= b.n[ax]) : (c.range[ax][1] < 0);
        if (!same) continue;
        for (int64_t l = c.range[ax][0]; l <= c.range[ax][1]; ++l)
          for (int64_t u = c.range[t1][0]; u <= c.range[t1][1]; ++u)
            for (int64_t w = c.range[t2][0]; w <= c.range[t2][1]; ++w) {
              const int64_t layer = hi ? l - b.n[ax] : -1 - l;
              cov[(size_t)(layer * b.n[t1] + u) * b.n[t2] + w] = 1;
            }
      }
      for (char v : cov)
        if (!v) {
          char m[160];
          std::snprintf(m, sizeof m, "region %d of block %d is connected but not every ghost cell has a donor",
                        region, bi);
          return fail(FVM_ERR_INVALID, m);
        }
    }
  }

  // -- layout of every live block
  int64_t need = 0;
  size_t max_cells = 0;
  for (int bi : live_blocks) {
    HBlock& b = blocks[bi];
    const int idim = cases[b.case_id].cfg.idimension;
    b.px = round_up(b.n[0] + kPadX + kGhost, 4);
    b.py = b.n[1] + 2 * kGhost;
    b.zpad = (idim == 3) ? kGhost : 0;
    b.pz = b.n[2] + 2 * b.zpad;
    b.sy = b.px;
    b.sz = b.px * b.py;
    b.org = kPadX + kGhost * b.sy + b.zpad * b.sz;
    b.padded = padded_cells(idim, b.n);
    need += b.padded;
    max_cells = std::max(max_cells, (size_t)(b.n[0] * b.n[1] * b.n[2]));
  }

  // -- the arena: created once (reserved size or exactly what is needed),
  //    grown only in the unreserved mode
  if (cap_ == 0) {
    nroles_ = (max_stages_ == 4) ? 4 : 3;
    const int64_t cap = round_up(std::max(reserved_, need), 64);
    if (cap >= ((int64_t)1 << 40)) return fail(FVM_ERR_INVALID, "grid too large");
    for (int r = 0; r < nroles_; ++r) {
      cudaError_t e = cudaMalloc(&role_[r], sizeof(double) * 5 * cap);
      if (e != cudaSuccess) return fail(FVM_ERR_NOMEM, std::string("state allocation: ") + cudaGetErrorString(e));
      CK(cudaMemsetAsync(role_[r], 0, sizeof(double) * 5 * cap, stream));
    }
    for (int r = nroles_; r < NROLE; ++r) role_[r] = role_[ROLE_A];
    cap_ = cap;
    free_.clear();
    free_.push_back({0, cap_});
  }
  if (any_ns && !visc_) {
    CK(cudaMalloc(&visc_, sizeof(double) * 5 * cap_));
    CK(cudaMemsetAsync(visc_, 0, sizeof(double) * 5 * cap_, stream));
  }
  for (int bi : live_blocks) {
    HBlock& b = blocks[bi];
    if (b.slab_off >= 0) continue;
    int64_t off = -1;
    if (alloc_range(b.padded, &off) != 0) {
      if (reserved_ > 0) return fail(FVM_ERR_NOMEM, "HBM budget exhausted: the reserved arena has no room");
      int rc = grow_arena(std::max(need, cap_ + cap_ / 2));
      if (rc) return rc;
      if (alloc_range(b.padded, &off) != 0) return fail(FVM_ERR_NOMEM, "arena allocation failed");
    }
    b.slab_off = off;
  }
  for (int bi : live_blocks) {
    HBlock& b = blocks[bi];
    if (!b.fresh) continue;
    for (int r = 0; r < nroles_; ++r)
      for (int v = 0; v < 5; ++v)
        CK(cudaMemsetAsync(role_[r] + b.slab_off + v * cap_, 0, sizeof(double) * b.padded, stream));
    if (visc_)
      for (int v = 0; v < 5; ++v)
        CK(cudaMemsetAsync(visc_ + b.slab_off + v * cap_, 0, sizeof(double) * b.padded, stream));
    if (cases[b.case_id].cfg.store_rhs && !b.rhs_dev) {
      const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
      CK(cudaMalloc(&b.rhs_dev, bytes));
      CK(cudaMemsetAsync(b.rhs_dev, 0, bytes, stream));
    }
    b.fresh = false;
  }
  if (sizeof(double) * 5 * max_cells > staging_bytes_) {
    if (d_staging_) cudaFree(d_staging_);
    d_staging_ = nullptr;
    staging_bytes_ = sizeof(double) * 5 * max_cells;
    CK(cudaMalloc(&d_staging_, staging_bytes_));
  }
  laid_out_ = true;
  return FVM_OK;
}

// A device buffer of at least n elements (1 if n is 0), grown by half again
// when it must grow; its contents are not kept.
template <class T>
static cudaError_t grow_buf(T** p, size_t* cap, size_t n) {
  n = std::max<size_t>(n, 1);
  if (*p && *cap >= n) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t c = n + n / 2;
  const cudaError_t e = cudaMalloc(p, sizeof(T) * c);
  if (e == cudaSuccess) *cap = c;
  return e;
}

int Engine::plan() {
  // the instantiated step graphs are kept: build_graph() updates them in
  // place when the new step has the same shape (no launch can use them
  // before the plan completes: planned_ stays false until then)
  if (graph_) cudaGraphDestroy(graph_);
  if (graphm_) cudaGraphDestroy(graphm_);
  graph_ = nullptr;
  graphm_ = nullptr;
  if (!laid_out_) {
    int rc = layout();
    if (rc) return rc;
  }
  std::vector<int> live_cases, live_blocks;
  for (size_t c = 0; c < cases.size(); ++c)
    if (!cases[c].dead) live_cases.push_back((int)c);
  for (size_t b = 0; b < blocks.size(); ++b)
    if (!blocks[b].dead) live_blocks.push_back((int)b);
  max_stages_ = cases[live_cases[0]].cfg.rk_stages;

  // -- groups (one per distinct kernel) and tasks
  groups.clear();
  std::vector<Task> tasks;
  std::vector<int> block_task0(blocks.size(), 0), block_ntask(blocks.size(), 0);
  for (int ci : live_cases) {
    HCase& hc = cases[ci];
    const fvm_config& c = hc.cfg;
    const int dim = c.idimension;
    const int prec = c.precision;
    const bool tb = c.reconstruct == FVM_RECON_WENO && c.compat == FVM_COMPAT_TEXTBOOK;
    int tile = hc.tile;
    if (tile < 0) {
      // heuristic (the autotuner measures instead): 16 x 8 on 128 threads
      // for the FP32 flux and FP64 forms in 3D; exact FP64, whose expression
      // trees need more registers, and every 2D case (a task is one plane,
      // so the wider tile's smaller halo share pays: 39 vs 49 us per step in
      // FP64 on 256^2) take the register-capped 32 x 8 variant when the
      // blocks are at least 32 wide, else 16 x 16 (exact) / 16 x 8
      int64_t minx = 1 << 30;
      for (int b : hc.blocks) minx = std::min(minx, blocks[b].n[0]);
      if (prec == FVM_PREC_FP64_EXACT)
        tile = minx >= 32 ? 2 : 1;
      else
        tile = (dim == 2 && minx >= 32) ? 2 : 3;
    }
    int gi = -1;
    for (size_t g = 0; g < groups.size(); ++g) {
      const Group& G = groups[g];
      if (G.prec == prec && G.dim == dim && G.recon == c.reconstruct && G.flux == c.flux_split && G.tb == tb &&
          G.tile == tile)
        gi = (int)g;
    }
    if (gi < 0) {
      Group G;
      G.prec = prec;
      G.dim = dim;
      G.recon = c.reconstruct;
      G.flux = c.flux_split;
      G.tb = tb;
      G.tile = tile;
      if (!lookup_stage_kernel(prec, dim, c.reconstruct, c.flux_split, tb, tile, &G.k))
        return fail(FVM_ERR_UNSUPPORTED, "no compiled stage kernel for this scheme combination");
      groups.push_back(G);
      gi = (int)groups.size() - 1;
    }
    hc.group = gi;
  }
  for (auto& G : groups) {
    int occ = -1;
    for (const auto& e : occ_cache_)
      if (e.first == G.k.fn) occ = e.second;
    if (occ < 0) {
      CK(cudaFuncSetAttribute(G.k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.k.smem));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, G.k.fn, G.k.threads, G.k.smem));
      occ_cache_.emplace_back(G.k.fn, occ);
    }
    if (occ < 1) return fail(FVM_ERR_UNSUPPORTED, "stage kernel does not fit on an SM");
    G.grid = occ * num_sms;
  }
  // Tasks grouped by kernel; inside a group, longest z range first so the
  // work queue finishes with the short tasks.
  for (size_t g = 0; g < groups.size(); ++g) {
    Group& G = groups[g];
    G.task_off = (int)tasks.size();
    std::vector<Task> gt;
    // z chunk of the group's cases without a tuned one: the length with the
    // lowest estimated queue makespan over all the group's tasks. A task of c
    // planes costs c plane-times plus the warm-up of its z window (WENO: 2
    // planes of z-only work, MUSCL 1) and its set-up; the queue of T tasks of
    // total cost S and longest cost M on the kernel's resident CTAs takes M
    // while T fits on them, else about S / CTAs + (M / 2) (CTAs / T): taken
    // longest first, the queue ends on short tasks, the more so the more
    // tasks each CTA takes (on the 64-case batch the estimate picks the
    // longest chunks, as measured best). Alone, a small case takes short
    // chunks to spread over the CTAs; in a large batch the warm-ups dominate
    // and the chunks grow. The estimate costs O(blocks) per candidate, so
    // the re-plans of a serving loop stay cheap. The state does not depend
    // on the tiling (only the residual norms' summation order does).
    int64_t L_auto = 0;
    if (G.dim == 3) {
      auto in_group = [&](int ci) { return cases[ci].group == (int)g; };
      const double ovh = G.recon == FVM_RECON_WENO ? 1.0 : (G.recon == FVM_RECON_MUSCL ? 0.65 : 0.35);
      struct QStat {
        double tasks = 0, sum = 0, mx = 0;
      };
      auto add_case = [&](const HCase& hc, int64_t L, QStat& q) {
        for (int bi : hc.blocks) {
          const HBlock& b = blocks[bi];
          const int64_t ncol = ((b.n[0] + G.k.tx - 1) / G.k.tx) * ((b.n[1] + G.k.ty - 1) / G.k.ty);
          const int64_t nc = std::max<int64_t>(1, (b.n[2] + L - 1) / L);  // equal_chunks
          const int64_t longest = b.n[2] / nc + (b.n[2] % nc ? 1 : 0);
          q.tasks += (double)(ncol * nc);
          q.sum += (double)ncol * ((double)b.n[2] + (double)nc * ovh);
          q.mx = std::max(q.mx, (double)longest + ovh);
        }
      };
      bool any_auto = false;
      QStat fixed;
      for (int ci : live_cases) {
        if (!in_group(ci)) continue;
        if (cases[ci].zchunk > 0)
          add_case(cases[ci], cases[ci].zchunk, fixed);
        else
          any_auto = true;
      }
      double best = 0.0;
      for (int64_t cand = 64; any_auto && cand >= 4; cand -= (cand > 16 ? 4 : 2)) {
        QStat q = fixed;
        for (int ci : live_cases)
          if (in_group(ci) && cases[ci].zchunk <= 0) add_case(cases[ci], cand, q);
        const double m = q.tasks <= G.grid ? q.mx : q.sum / G.grid + 0.5 * q.mx * G.grid / q.tasks;
        if (L_auto <= 0 || m < best * 0.995) {
          best = m;
          L_auto = cand;
        }
      }
    }
    for (int ci : live_cases) {
      HCase& hc = cases[ci];
      if (hc.group != (int)g) continue;
      const int64_t L = hc.zchunk > 0 ? (int64_t)hc.zchunk : L_auto;
      std::vector<int64_t> z0s;
      std::vector<Task> ct;
      for (int bi : hc.blocks) {
        const HBlock& b = blocks[bi];
        if (G.dim == 3)
          equal_chunks(b.n[2], L, z0s);
        else
          z0s = {0, b.n[2]};
        for (size_t c = 0; c + 1 < z0s.size(); ++c)
          for (int64_t y0 = 0; y0 < b.n[1]; y0 += G.k.ty)
            for (int64_t x0 = 0; x0 < b.n[0]; x0 += G.k.tx) {
              Task t;
              t.blk = bi;
              t.x0 = (int)x0;
              t.y0 = (int)y0;
              t.z0 = (int)z0s[c];
              t.z1 = (int)z0s[c + 1];
              t.slot = 0;
              ct.push_back(t);
            }
      }
      // Tail split: when the case's tasks fill the queue's slots (resident
      // CTAs) k times and r more, its r shortest tasks are cut along z into
      // tail_split pieces, so the last, partial round of the queue runs on
      // more CTAs for a shorter time (each piece warms up its own z window).
      // It depends on the case and the kernel's slot count only, so a case
      // is tiled alike alone and batched.
      if (G.dim == 3 && hc.tail_split > 1 && (int64_t)ct.size() > G.grid) {
        std::stable_sort(ct.begin(), ct.end(),
                         [](const Task& a, const Task& b) { return (a.z1 - a.z0) > (b.z1 - b.z0); });
        const size_t r = ct.size() % (size_t)G.grid;
        std::vector<Task> pieces;
        for (size_t i = ct.size() - r; i < ct.size(); ++i) {
          const Task& t = ct[i];
          const int n = t.z1 - t.z0;
          const int sp = std::min(hc.tail_split, n / 2);  // pieces of at least 2 planes
          for (int q = 0; q < std::max(sp, 1); ++q) {
            Task u = t;
            if (sp > 1) {
              u.z0 = t.z0 + (int)((int64_t)n * q / sp);
              u.z1 = t.z0 + (int)((int64_t)n * (q + 1) / sp);
            }
            pieces.push_back(u);
          }
        }
        ct.resize(ct.size() - r);
        ct.insert(ct.end(), pieces.begin(), pieces.end());
      }
      gt.insert(gt.end(), ct.begin(), ct.end());
    }
    std::stable_sort(gt.begin(), gt.end(), [](const Task& a, const Task& b) { return (a.z1 - a.z0) > (b.z1 - b.z0); });
    tasks.insert(tasks.end(), gt.begin(), gt.end());
    G.ntasks = (int)tasks.size() - G.task_off;
    G.grid = std::max(1, std::min(G.grid, G.ntasks));
  }
  // partial slots: contiguous per block (the finalize sums a block's slots)
  {
    std::vector<std::vector<int>> per_block(blocks.size());
    for (size_t t = 0; t < tasks.size(); ++t) per_block[tasks[t].blk].push_back((int)t);
    int slot = 0;
    for (int bi : live_blocks) {
      block_task0[bi] = slot;
      block_ntask[bi] = (int)per_block[bi].size();
      for (int t : per_block[bi]) tasks[t].slot = slot++;
    }
  }
  ntasks_total = (int64_t)tasks.size();

  // -- viscous task lists, one per (precision form, dimension): Navier-Stokes
  // blocks in column tiles over equal z chunks. The kernel is
  // throughput-bound per SM (its CTAs share the SM's shared-memory pipe), so
  // a 3D chunk length is scored by the largest per-SM sum of task costs
  // (longest-first onto the SMs) over the CTAs an SM holds, but no less than
  // half the longest task (an SM left with one task runs it at most about
  // twice as fast). A task of c planes costs c plane-times plus its prologue
  // (two extra planes converted, one extra z face).
  for (int prec = 0; prec < 3; ++prec) {
    for (int dim : {3, 2}) {
      const int li = prec * 2 + (dim == 3 ? 0 : 1);
      const int64_t vtx = visc_tx(prec), vty = visc_ty(prec);
      vlist_off_[li] = (int)tasks.size();
      std::vector<const HBlock*> ns;
      for (int bi : live_blocks) {
        const fvm_config& c = cases[blocks[bi].case_id].cfg;
        if (c.equation == FVM_EQ_NAVIER_STOKES && c.idimension == dim && c.precision == prec)
          ns.push_back(&blocks[bi]);
      }
      int64_t vz = 16;
      std::vector<int64_t> z0s;
      if (dim == 3 && !ns.empty()) {
        int occ = 1;
        CK(visc_occupancy(prec, &occ));
        double best = 0.0;
        std::vector<double> cost;
        for (int64_t cand = 64; cand >= 4; cand -= (cand > 16 ? 4 : 2)) {
          cost.clear();
          double longest = 0.0;
          for (const HBlock* b : ns) {
            const int64_t ncol = ((b->n[0] + vtx - 1) / vtx) * ((b->n[1] + vty - 1) / vty);
            equal_chunks(b->n[2], cand, z0s);
            for (size_t c = 0; c + 1 < z0s.size(); ++c)
              for (int64_t q = 0; q < ncol; ++q) {
                cost.push_back((double)(z0s[c + 1] - z0s[c]) + 1.5);
                longest = std::max(longest, cost.back());
              }
          }
          const double m = std::max(queue_makespan(cost, num_sms) / occ, 0.5 * longest);
          if (best <= 0.0 || m < best * 0.995) {
            best = m;
            vz = cand;
          }
        }
      }
      for (const HBlock* b : ns) {
        const int bi = (int)(b - blocks.data());
        if (dim == 3)
          equal_chunks(b->n[2], vz, z0s);
        else
          z0s = {0, b->n[2]};
        for (size_t ch = 0; ch + 1 < z0s.size(); ++ch)
          for (int64_t y0 = 0; y0 < b->n[1]; y0 += vty)
            for (int64_t x0 = 0; x0 < b->n[0]; x0 += vtx) {
              Task t;
              t.blk = bi;
              t.x0 = (int)x0;
              t.y0 = (int)y0;
              t.z0 = (int)z0s[ch];
              t.z1 = (int)z0s[ch + 1];
              t.slot = 0;
              tasks.push_back(t);
            }
      }
      vlist_n_[li] = (int)tasks.size() - vlist_off_[li];
    }
  }

  // -- ghost gather pairs (slab element offsets). A case's pairs depend only
  //    on its own blocks (connections never cross cases) and their arena
  //    offsets, which never change while the case lives, so they are built
  //    once per case and reused by every later re-plan (the serving loop
  //    re-plans at each admission and retirement). Cell offsets within a role
  //    slab stay below 2^31 (a slab of 2^31 cells would take 344 GB in the 4
  //    roles, twice the HBM): 8 bytes per pair.
  if (cap_ >= ((int64_t)1 << 31)) return fail(FVM_ERR_INVALID, "arena too large for 32-bit ghost offsets");
  std::vector<int32_t> cp;  // pairs of the case being built
  auto add_pair = [&](int bi, const int64_t x[3]) -> int {
    int64_t y[3] = {x[0], x[1], x[2]};
    int src_blk = -1;
    if (resolve(bi, y, &src_blk) != 0) return -1;
    const HBlock& b = blocks[bi];
    const HBlock& s = blocks[src_blk];
    cp.push_back((int32_t)(b.slab_off + b.org + x[0] + x[1] * b.sy + x[2] * b.sz));
    cp.push_back((int32_t)(s.slab_off + s.org + y[0] + y[1] * s.sy + y[2] * s.sz));
    return 0;
  };
  // One connection's ghost cells. When the connection's range lies wholly
  // outside the block along one axis and wholly inside along the others, in
  // a region that is not transmissive, no earlier connection of the block
  // overlaps it, and its image under the donor map is all real donor cells,
  // resolve() would take exactly one hop through this connection for every
  // cell: the pairs are then the affine map itself, row by row.
  auto add_conn = [&](int bi, size_t ci) -> int {
    const HBlock& b = blocks[bi];
    const HConn& c = b.conns[ci];
    int out = 0, inside = 0, region = 0;
    for (int d = 0; d < 3; ++d) {
      if (c.range[d][1] < 0) {
        ++out;
        region = 2 * d + 1;
      } else if (c.range[d][0] >= b.n[d]) {
        ++out;
        region = 2 * d + 2;
      } else if (c.range[d][0] >= 0 && c.range[d][1] < b.n[d]) {
        ++inside;
      }
    }
    bool direct = out == 1 && inside == 2 && b.bc[region - 1] != FVM_BC_TRANSMISSIVE;
    for (size_t e = 0; e < ci && direct; ++e) {
      const HConn& o = b.conns[e];
      bool ov = true;
      for (int d = 0; d < 3; ++d) ov = ov && o.range[d][0] <= c.range[d][1] && c.range[d][0] <= o.range[d][1];
      direct = !ov;
    }
    const HBlock& s = blocks[c.donor];
    int64_t ys[3] = {0, 0, 0};  // donor offset step per unit step of x along each axis
    int64_t y0[3];
    const int64_t sst[3] = {1, s.sy, s.sz};
    for (int d = 0; d < 3 && direct; ++d) {
      const int dd = std::abs(c.dtype[d]) - 1;
      const int64_t sg = c.dtype[d] > 0 ? 1 : -1;
      const int64_t a0 = c.drange[d][0], a1 = c.drange[d][0] + sg * (c.range[d][1] - c.range[d][0]);
      direct = std::min(a0, a1) >= 0 && std::max(a0, a1) < s.n[dd];
      y0[dd] = a0;
      ys[d] = sg * sst[dd];
    }
    if (direct) {
      const int64_t src0 = s.slab_off + s.org + y0[0] + y0[1] * s.sy + y0[2] * s.sz;
      const int64_t dst0 = b.slab_off + b.org;
      const int64_t ni = c.range[0][1] - c.range[0][0] + 1;
      for (int64_t k = c.range[2][0]; k <= c.range[2][1]; ++k)
        for (int64_t j = c.range[1][0]; j <= c.range[1][1]; ++j) {
          int64_t dst = dst0 + c.range[0][0] + j * b.sy + k * b.sz;
          int64_t src = src0 + (j - c.range[1][0]) * ys[1] + (k - c.range[2][0]) * ys[2];
          for (int64_t i = 0; i < ni; ++i, ++dst, src += ys[0]) {
            cp.push_back((int32_t)dst);
            cp.push_back((int32_t)src);
          }
        }
      return 0;
    }
    for (int64_t k = c.range[2][0]; k <= c.range[2][1]; ++k)
      for (int64_t j = c.range[1][0]; j <= c.range[1][1]; ++j)
        for (int64_t i = c.range[0][0]; i <= c.range[0][1]; ++i) {
          const int64_t x[3] = {i, j, k};
          if (add_pair(bi, x) != 0) return -1;
        }
    return 0;
  };
  int64_t npairs_total = 0;
  for (int ci : live_cases) {
    HCase& hc = cases[ci];
    std::vector<int64_t> key;
    for (int bi : hc.blocks) key.push_back(blocks[bi].slab_off);
    if (!hc.pairs_valid || key != hc.pairs_key) {
      cp.clear();
      for (int bi : hc.blocks) {
        const HBlock& b = blocks[bi];
        for (size_t c = 0; c < b.conns.size(); ++c)
          if (add_conn(bi, c) != 0) return fail(FVM_ERR_INVALID, "ghost cell without a real donor");
        if (hc.cfg.equation == FVM_EQ_NAVIER_STOKES) {
          // layer-1 edge ghosts read by the viscous stencil where both regions
          // are connected (a transmissive axis is clamped on load instead)
          const int idim = hc.cfg.idimension;
          for (int a = 0; a < idim; ++a)
            for (int a2 = a + 1; a2 < idim; ++a2) {
              const int c3 = 3 - a - a2;
              for (int sa = 0; sa < 2; ++sa)
                for (int sb = 0; sb < 2; ++sb) {
                  if (b.bc[2 * a + sa] == FVM_BC_TRANSMISSIVE || b.bc[2 * a2 + sb] == FVM_BC_TRANSMISSIVE) continue;
                  for (int64_t t = 0; t < b.n[c3]; ++t) {
                    int64_t x[3];
                    x[a] = sa ? b.n[a] : -1;
                    x[a2] = sb ? b.n[a2] : -1;
                    x[c3] = t;
                    if (add_pair(bi, x) != 0) return fail(FVM_ERR_INVALID, "edge ghost without a real donor");
                  }
                }
            }
        }
      }
      hc.pairs_cache = cp;
      hc.pairs_key = key;
      hc.pairs_valid = true;
      hc.pairs_dev_off = -1;
    }
    npairs_total += (int64_t)hc.pairs_cache.size() / 2;
  }
  npairs = npairs_total;

  // -- device descriptors (dead blocks keep an empty descriptor)
  h_dblocks_.assign(blocks.size(), DevBlock());
  for (size_t bi = 0; bi < blocks.size(); ++bi) {
    DevBlock& d = h_dblocks_[bi];
    std::memset(&d, 0, sizeof d);
    const HBlock& b = blocks[bi];
    d.case_id = b.case_id;
    if (b.dead) continue;
    for (int r = 0; r < NROLE; ++r) d.q[r] = role_[r] + b.slab_off + b.org;
    d.rhs = b.rhs_dev;
    d.visc = (visc_ && cases[b.case_id].cfg.equation == FVM_EQ_NAVIER_STOKES) ? visc_ + b.slab_off + b.org : nullptr;
    d.vs = cap_;
    for (int a = 0; a < 3; ++a) {
      d.n[a] = (int32_t)b.n[a];
      d.dr[a] = b.dr[a];
      d.inv_dr[a] = 1.0 / b.dr[a];
    }
    d.sy = (int32_t)b.sy;
    d.sz = (int32_t)b.sz;
    int mask = 0;
    for (int r = 0; r < 6; ++r)
      if (b.bc[r] != FVM_BC_TRANSMISSIVE) mask |= 1 << r;
    d.ghost_mask = mask;
    d.task0 = block_task0[bi];
    d.ntask = block_ntask[bi];
  }
  std::vector<DevCase> hcases(cases.size());
  std::vector<int> case_blk;
  for (size_t ci = 0; ci < cases.size(); ++ci) {
    const fvm_config& c = cases[ci].cfg;
    DevCase& d = hcases[ci];
    std::memset(&d, 0, sizeof d);
    d.gamma = c.gamma;
    d.gm1 = c.gamma - 1.0;
    d.kappa = c.kappa;
    d.entropy_fix = c.entropy_fix;
    d.cfl = c.cfl;
    d.dt_fixed = c.dt;
    d.mu = c.mu;
    d.prandtl = c.prandtl;
    d.kq = c.mu * c.gamma / (c.prandtl * (c.gamma - 1.0));
    d.limiter = c.limiter;
    d.compat = c.compat;
    d.timestep_set = c.timestep_set;
    d.idim = c.idimension;
    d.rk_stages = c.rk_stages;
    d.equation = c.equation;
    d.store_rhs = c.store_rhs;
    d.precision = c.precision;
    d.block0 = (int)case_blk.size();
    d.nblocks = 0;
    if (cases[ci].dead) continue;
    for (int b : cases[ci].blocks) case_blk.push_back(b);
    d.nblocks = (int)cases[ci].blocks.size();
  }
  // per-case evolving state: kept across re-plans, initialised for new cases
  if (state_cap_ < (int)cases.size()) {
    const int ncap = std::max<int>(64, (int)cases.size() * 2);
    DevCaseState* ns = nullptr;
    CK(cudaMalloc(&ns, sizeof(DevCaseState) * ncap));
    CK(cudaMemsetAsync(ns, 0, sizeof(DevCaseState) * ncap, stream));
    if (d_state_) {
      CK(cudaMemcpyAsync(ns, d_state_, sizeof(DevCaseState) * state_cap_, cudaMemcpyDeviceToDevice, stream));
      CK(cudaStreamSynchronize(stream));
      cudaFree(d_state_);
    }
    d_state_ = ns;
    state_cap_ = ncap;
  }
  for (int ci : live_cases) {
    if (!cases[ci].fresh) continue;
    DevCaseState s;
    std::memset(&s, 0, sizeof s);
    s.dt = cases[ci].cfg.dt;
    CK(cudaMemcpyAsync(d_state_ + ci, &s, sizeof s, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    cases[ci].fresh = false;
    cases[ci].dt_stale = true;
  }
  // Descriptor buffers grow (never shrink) across re-plans, so admitting or
  // retiring a case between steps costs no cudaFree / cudaMalloc (which
  // would synchronise the device) unless a buffer must grow; a growth frees
  // the old buffer and clears its pointer first, so a failed allocation
  // leaves a null member, never a freed address.
  planned_ = false;
  ncounters_ = max_stages_ * (int)groups.size();
  CK(grow_buf(&d_blocks_, &cap_blocks_, blocks.size()));
  CK(grow_buf(&d_cases_, &cap_cases_, cases.size()));
  CK(grow_buf(&d_case_blk_, &cap_case_blk_, case_blk.size()));
  CK(grow_buf(&d_tasks_, &cap_tasks_, tasks.size()));
  CK(grow_buf(&d_partials_, &cap_partials_, kPartStride * std::max<size_t>(1, tasks.size())));
  CK(grow_buf(&d_pairs_alt_, &cap_pairs_alt_, std::max<size_t>(2, 2 * (size_t)npairs)));
  CK(grow_buf(&d_counters_, &cap_counters_, (size_t)std::max(1, ncounters_)));
  CK(grow_buf(&d_casemax_, &cap_casemax_, cases.size()));
  CK(cudaMemcpyAsync(d_blocks_, h_dblocks_.data(), sizeof(DevBlock) * blocks.size(), cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_cases_, hcases.data(), sizeof(DevCase) * cases.size(), cudaMemcpyHostToDevice, stream));
  if (!case_blk.empty())
    CK(cudaMemcpyAsync(d_case_blk_, case_blk.data(), sizeof(int) * case_blk.size(), cudaMemcpyHostToDevice, stream));
  if (!tasks.empty())
    CK(cudaMemcpyAsync(d_tasks_, tasks.data(), sizeof(Task) * tasks.size(), cudaMemcpyHostToDevice, stream));
  // the pair array is assembled on the device: a case already there moves
  // by a device copy, only a new case's pairs cross from the host (the
  // offsets are taken over once every copy is enqueued)
  {
    std::vector<int64_t> offs(live_cases.size(), -1);
    int64_t off = 0;
    for (size_t i = 0; i < live_cases.size(); ++i) {
      const HCase& hc = cases[live_cases[i]];
      const int64_t n = (int64_t)hc.pairs_cache.size();
      if (n == 0) continue;
      if (hc.pairs_dev_off >= 0)
        CK(cudaMemcpyAsync(d_pairs_alt_ + off, d_pairs_ + hc.pairs_dev_off, sizeof(int32_t) * n,
                           cudaMemcpyDeviceToDevice, stream));
      else
        CK(cudaMemcpyAsync(d_pairs_alt_ + off, hc.pairs_cache.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                           stream));
      offs[i] = off;
      off += n;
    }
    for (size_t i = 0; i < live_cases.size(); ++i) cases[live_cases[i]].pairs_dev_off = offs[i];
    std::swap(d_pairs_, d_pairs_alt_);
    std::swap(cap_pairs_, cap_pairs_alt_);
  }
  CK(cudaMemsetAsync(d_counters_, 0, sizeof(int) * std::max(1, ncounters_), stream));
  CK(cudaMemsetAsync(d_partials_, 0, sizeof(double) * kPartStride * std::max<size_t>(1, tasks.size()), stream));

  // -- tensor maps of the groups whose kernel prefetches with TMA: per block
  //    and input role (A, B, C), the plane box and the z box over the block's
  //    padded box as a 4D tensor (x, y, z, variable)
  //    (grow-only device buffers, one per group slot; a block's maps are
  //    encoded once for its arena place and box shape and kept across
  //    re-plans, so admitting a case encodes only its own blocks)
  if (d_tmap_.size() < groups.size()) {
    d_tmap_.resize(groups.size(), nullptr);
    cap_tmap_.resize(groups.size(), 0);
  }
  if (!d_err_) CK(cudaMalloc(&d_err_, sizeof(int32_t)));
  CK(cudaMemsetAsync(d_err_, 0, sizeof(int32_t), stream));
  std::vector<CUtensorMap> maps;
  for (size_t g = 0; g < groups.size(); ++g) {
    const Group& G = groups[g];
    if (!G.k.tma) continue;
    PFN_cuTensorMapEncodeTiled enc = encode_fn();
    if (!enc) return fail(FVM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    maps.assign(blocks.size() * NROLE * 2, CUtensorMap());
    std::memset(maps.data(), 0, sizeof(CUtensorMap) * maps.size());
    for (int ci : live_cases) {
      if (cases[ci].group != (int)g) continue;
      for (int bi : cases[ci].blocks) {
        HBlock& b = blocks[bi];
        const int64_t key[4] = {(int64_t)(uintptr_t)role_[0], cap_, b.slab_off,
                                (int64_t)G.k.box_w | ((int64_t)G.k.box_h << 16) | ((int64_t)G.k.tx << 32) |
                                    ((int64_t)G.k.ty << 48)};
        if (b.tmaps.size() != (size_t)NROLE * 2 || !std::equal(key, key + 4, b.tmap_key)) {
          b.tmaps.assign((size_t)NROLE * 2, CUtensorMap());
          const cuuint64_t dims[4] = {(cuuint64_t)b.px, (cuuint64_t)b.py, (cuuint64_t)b.pz, 5};
          const cuuint64_t strides[3] = {(cuuint64_t)(b.sy * 8), (cuuint64_t)(b.sz * 8), (cuuint64_t)(cap_ * 8)};
          const cuuint32_t box_p[4] = {(cuuint32_t)G.k.box_w, (cuuint32_t)G.k.box_h, 1, 5};
          const cuuint32_t box_z[4] = {(cuuint32_t)G.k.tx, (cuuint32_t)G.k.ty, 1, 5};
          const cuuint32_t estr[4] = {1, 1, 1, 1};
          for (int r = 0; r < NROLE; ++r) {
            void* base = role_[r] + b.slab_off;
            for (int w = 0; w < 2; ++w) {
              const CUresult e = enc(&b.tmaps[(size_t)r * 2 + w], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims,
                                     strides, w == 0 ? box_p : box_z, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
              if (e != CUDA_SUCCESS) {
                b.tmaps.clear();
                return fail(FVM_ERR_CUDA, "cuTensorMapEncodeTiled failed for a block");
              }
            }
          }
          std::copy(key, key + 4, b.tmap_key);
        }
        std::copy(b.tmaps.begin(), b.tmaps.end(), maps.begin() + (size_t)bi * NROLE * 2);
      }
    }
    CK(grow_buf(&d_tmap_[g], &cap_tmap_[g], maps.size()));
    CK(cudaMemcpyAsync(d_tmap_[g], maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, stream));
  }
  CK(cudaStreamSynchronize(stream));
  planned_ = true;
  prepared_ = false;
  return build_graph();
}

// Enqueue one full time step on `stream`: per stage the optional viscous
// kernel, one fused stage launch per scheme group and the ghost gather; then
// the finalize. With `evs`, an event is recorded after every launch and the
// kind of each launch (1 stage, 2 gather, 3 viscous, 4 finalize) returned.
StageArgs Engine::stage_args(int g, int m) const {
  const Group& G = groups[g];
  const int S = max_stages_;
  int rin, rout;
  stage_roles(S, m, &rin, &rout);
  StageArgs a;
  a.tasks = d_tasks_ + G.task_off;
  a.ntasks = G.ntasks;
  a.counter = d_counters_ + (m - 1) * (int)groups.size() + g;
  a.blocks = d_blocks_;
  a.cases = d_cases_;
  a.cstate = d_state_;
  a.partials = d_partials_;
  a.m = m;
  a.rin = rin;
  a.rout = rout;
  a.rq0 = ROLE_A;
  a.racc = (S == 4) ? ROLE_ACC : ROLE_A;
  a.last = (m == S) ? 1 : 0;
  a.tmap = d_tmap_[g];
  a.err = d_err_;
  a.drop_copies = drop_copies_ ? 1 : 0;
  return a;
}

int Engine::enqueue_step(cudaEvent_t* evs, int nev, int* kinds, int* nlaunch) {
  const int S = max_stages_;
  // groups run as parallel branches of the captured graph (fork / join on
  // side streams); the profiled path launches them in sequence to time each
  const bool fork = (evs == nullptr) && groups.size() > 1;
  // a single-group step graph chains its kernels by programmatic dependent
  // launch: each launch's CTAs are scheduled while its predecessor drains
  // (every step kernel begins with pdl_wait)
  const bool pdl = (evs == nullptr) && !fork;
  int n = 0;
  auto mark = [&](int kind) -> cudaError_t {
    if (evs && n < nev) {
      kinds[n] = kind;
      cudaError_t e = cudaEventRecord(evs[n + 1], stream);
      ++n;
      return e;
    }
    ++n;
    return cudaSuccess;
  };
  if (evs && nev > 0) CK(cudaEventRecord(evs[0], stream));
  int ev_i = 0;
  for (int m = 1; m <= S; ++m) {
    int rin, rout;
    stage_roles(S, m, &rin, &rout);
    for (int li = 0; li < 6; ++li) {
      if (vlist_n_[li] == 0) continue;
      CK(launch_visc(d_blocks_, d_cases_, d_tasks_ + vlist_off_[li], vlist_n_[li], li % 2 == 0 ? 3 : 2, li / 2,
                     rin, stream, pdl));
      CK(mark(3));
    }
    if (fork) CK(cudaEventRecord(fork_ev_[ev_i], stream));
    const int fork_ev = ev_i++;
    for (size_t g = 0; g < groups.size(); ++g) {
      const Group& G = groups[g];
      StageArgs a = stage_args((int)g, m);
      void* args[] = {&a};
      cudaStream_t st = stream;
      if (fork) {
        st = side_[g];
        CK(cudaStreamWaitEvent(st, fork_ev_[fork_ev], 0));
      }
      LaunchCfg L(dim3(G.grid), dim3(G.k.threads), G.k.smem, st, pdl);
      CK(cudaLaunchKernelExC(&L.cfg, G.k.fn, args));
      if (fork) {
        CK(cudaEventRecord(fork_ev_[ev_i], st));
        CK(cudaStreamWaitEvent(stream, fork_ev_[ev_i], 0));
        ++ev_i;
      }
      CK(mark(1));
    }
    if (npairs > 0) {
      CK(launch_gather(role_[rout], cap_, d_pairs_, npairs, stream, pdl));
      CK(mark(2));
    }
  }
  CK(launch_finalize(d_blocks_, d_cases_, d_case_blk_, d_state_, (int)cases.size(), d_partials_, d_counters_,
                     ncounters_, stream, pdl));
  CK(mark(4));
  if (nlaunch) *nlaunch = n;
  return FVM_OK;
}

void Engine::destroy_graphs() {
  if (gexec_) cudaGraphExecDestroy(gexec_);
  if (graph_) cudaGraphDestroy(graph_);
  if (gexecm_) cudaGraphExecDestroy(gexecm_);
  if (graphm_) cudaGraphDestroy(graphm_);
  gexec_ = nullptr;
  graph_ = nullptr;
  gexecm_ = nullptr;
  graphm_ = nullptr;
}

// nsteps steps: runs of kMultiSteps from the multi-step graph, the rest one
// by one.
cudaError_t Engine::launch_steps(int nsteps) {
  int n = nsteps;
  for (; gexecm_ && n >= kMultiSteps; n -= kMultiSteps) {
    cudaError_t e = cudaGraphLaunch(gexecm_, stream);
    if (e != cudaSuccess) return e;
  }
  for (; n > 0; --n) {
    cudaError_t e = cudaGraphLaunch(gexec_, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Capture one time step (and kMultiSteps of them) and make them launchable:
// an instantiated graph of an earlier plan is updated in place when the new
// capture has its shape (same kernels and dependencies: a serving engine
// admitting or retiring cases of the same schemes), which costs a fraction of
// a new instantiation; otherwise it is instantiated again.
int Engine::build_graph() {
  while (side_.size() < groups.size()) {
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    side_.push_back(st);
  }
  const size_t nev = (size_t)max_stages_ * (groups.size() + 1);
  while (fork_ev_.size() < nev) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    fork_ev_.push_back(e);
  }
  auto capture = [&](int nsteps, int* launches, cudaGraph_t* out) -> int {
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    for (int i = 0; i < nsteps && rc == 0; ++i) rc = enqueue_step(nullptr, 0, nullptr, i == 0 ? launches : nullptr);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    *out = g;
    return FVM_OK;
  };
  auto make_exec = [&](cudaGraph_t g, cudaGraphExec_t* exec) -> int {
    if (*exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(*exec, g, &info) == cudaSuccess) return FVM_OK;
      (void)cudaGetLastError();  // a different shape: instantiate anew
      cudaGraphExecDestroy(*exec);
      *exec = nullptr;
    }
    CK(cudaGraphInstantiate(exec, g, 0));
    return FVM_OK;
  };
  int launches = 0;
  int rc = capture(1, &launches, &graph_);
  if (!rc) rc = make_exec(graph_, &gexec_);
  if (rc) return rc;
  kernel_launches_per_step = launches;
  rc = capture(kMultiSteps, nullptr, &graphm_);
  if (!rc) rc = make_exec(graphm_, &gexecm_);
  return rc;
}

int Engine::profile_step(float* ms, int* kinds, int cap, int* n) {
  int rc = ensure_planned();
  if (rc) return rc;
  if (!prepared_) {
    rc = prepare();
    if (rc) return rc;
  }
  const int nev = kernel_launches_per_step + 1;
  std::vector<cudaEvent_t> ev(nev);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<int> k(nev, 0);
  int nl = 0;
  rc = enqueue_step(ev.data(), nev - 1, k.data(), &nl);
  if (rc) return rc;
  CK(cudaEventSynchronize(ev[nev - 1]));
  const int m = std::min(cap, nl);
  for (int i = 0; i < m; ++i) {
    CK(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
    kinds[i] = k[i];
  }
  for (auto& e : ev) cudaEventDestroy(e);
  *n = m;
  return FVM_OK;
}

int Engine::prepare() {
  int rc = ensure_planned();
  if (rc) return rc;
  if (npairs > 0) CK(launch_gather(role_[ROLE_A], cap_, d_pairs_, npairs, stream));
  // dt from the state only for cases whose state was uploaded since their
  // last step (or that are new); a running case keeps the dt its last step
  // computed, so adding or removing other cases does not change its results
  std::vector<int> mask(cases.size(), 0);
  bool any = false;
  for (size_t c = 0; c < cases.size(); ++c)
    if (!cases[c].dead && cases[c].dt_stale) mask[c] = 1, any = true;
  if (any) {
    if (dtmask_cap_ < (int)cases.size()) {
      if (d_dtmask_) cudaFree(d_dtmask_);
      d_dtmask_ = nullptr;
      CK(cudaMalloc(&d_dtmask_, sizeof(int) * cases.size()));
      dtmask_cap_ = (int)cases.size();
    }
    CK(cudaMemcpyAsync(d_dtmask_, mask.data(), sizeof(int) * cases.size(), cudaMemcpyHostToDevice, stream));
    CK(launch_init_dt(d_blocks_, (int)blocks.size(), d_cases_, d_state_, (int)cases.size(), d_casemax_, d_dtmask_,
                      ROLE_A, stream));
    CK(cudaStreamSynchronize(stream));  // the mask's host copy goes out of scope
    for (auto& c : cases) c.dt_stale = false;
  }
  prepared_ = true;
  return FVM_OK;
}

// ---------------------------------------------------------------- state
int Engine::set_state(int blk, const double* q) {
  if (!live_block(blk)) return fail(FVM_ERR_INVALID, "bad block id");
  if (!q) return fail(FVM_ERR_INVALID, "null state");
  if (!laid_out_) {
    int rc = layout();
    if (rc) return rc;
  }
  const HBlock& b = blocks[blk];
  const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
  CK(cudaMemcpyAsync(d_staging_, q, bytes, cudaMemcpyHostToDevice, stream));
  CK(launch_unpack(role_[ROLE_A] + b.slab_off + b.org, cap_, (int)b.sy, (int)b.sz, (int)b.n[0], (int)b.n[1], (int)b.n[2],
                   d_staging_, stream));
  cases[b.case_id].dt_stale = true;
  // a new state clears the case's error status (NaN / divergence of an
  // earlier state)
  if (d_state_ && b.case_id < state_cap_ && !cases[b.case_id].fresh)
    CK(cudaMemsetAsync(reinterpret_cast<char*>(d_state_ + b.case_id) + offsetof(DevCaseState, status), 0,
                       sizeof(int32_t), stream));
  CK(cudaStreamSynchronize(stream));
  prepared_ = false;
  return FVM_OK;
}

int Engine::get_state(int blk, double* q, int prim) {
  if (!live_block(blk)) return fail(FVM_ERR_INVALID, "bad block id");
  if (!q) return fail(FVM_ERR_INVALID, "null output");
  if (!laid_out_) {
    if (cap_ == 0) return fail(FVM_ERR_STATE, "no state uploaded yet");
    int rc = layout();
    if (rc) return rc;
  }
  const HBlock& b = blocks[blk];
  const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
  CK(launch_pack(role_[ROLE_A] + b.slab_off + b.org, cap_, (int)b.sy, (int)b.sz, (int)b.n[0], (int)b.n[1], (int)b.n[2],
                 d_staging_, prim, cases[b.case_id].cfg.gamma - 1.0, stream));
  CK(cudaMemcpyAsync(q, d_staging_, bytes, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return FVM_OK;
}

// The second staging buffer, the copy stream and its events, made on first
// use of set_states / get_states.
int Engine::ensure_xfer() {
  if (staging2_bytes_ < staging_bytes_) {
    if (d_staging2_) cudaFree(d_staging2_);
    d_staging2_ = nullptr;
    staging2_bytes_ = 0;
    CK(cudaMalloc(&d_staging2_, staging_bytes_));
    staging2_bytes_ = staging_bytes_;
  }
  if (!xstream_) CK(cudaStreamCreateWithFlags(&xstream_, cudaStreamNonBlocking));
  for (auto& e : xev_)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return FVM_OK;
}

// fvm_set_state for n blocks: block i goes through staging buffer i % 2; its
// host-to-device copy (on xstream_) waits only for the unpack of block i - 2,
// so the copies run back to back while the engine stream unpacks. One
// synchronisation at the end: the host buffers are not read after return.
int Engine::set_states(int n, const int* blk, const double* const* q) {
  if (n < 0 || (n > 0 && (!blk || !q))) return fail(FVM_ERR_INVALID, "bad block list");
  for (int i = 0; i < n; ++i) {
    if (!live_block(blk[i])) return fail(FVM_ERR_INVALID, "bad block id");
    if (!q[i]) return fail(FVM_ERR_INVALID, "null state");
  }
  if (n == 0) return FVM_OK;
  if (!laid_out_) {
    int rc = layout();
    if (rc) return rc;
  }
  int rc = ensure_xfer();
  if (rc) return rc;
  double* stg[2] = {d_staging_, d_staging2_};
  cudaEvent_t* copied = xev_;
  cudaEvent_t* used = xev_ + 2;
  CK(cudaEventRecord(xev_[4], stream));  // earlier work on the engine stream may read the staging buffers
  CK(cudaStreamWaitEvent(xstream_, xev_[4], 0));
  for (int i = 0; i < n; ++i) {
    const int j = i & 1;
    const HBlock& b = blocks[blk[i]];
    const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
    if (i >= 2) CK(cudaStreamWaitEvent(xstream_, used[j], 0));
    CK(cudaMemcpyAsync(stg[j], q[i], bytes, cudaMemcpyHostToDevice, xstream_));
    CK(cudaEventRecord(copied[j], xstream_));
    CK(cudaStreamWaitEvent(stream, copied[j], 0));
    CK(launch_unpack(role_[ROLE_A] + b.slab_off + b.org, cap_, (int)b.sy, (int)b.sz, (int)b.n[0], (int)b.n[1],
                     (int)b.n[2], stg[j], stream));
    CK(cudaEventRecord(used[j], stream));
    cases[b.case_id].dt_stale = true;
    if (d_state_ && b.case_id < state_cap_ && !cases[b.case_id].fresh)
      CK(cudaMemsetAsync(reinterpret_cast<char*>(d_state_ + b.case_id) + offsetof(DevCaseState, status), 0,
                         sizeof(int32_t), stream));
  }
  CK(cudaStreamSynchronize(stream));
  prepared_ = false;
  return FVM_OK;
}

// fvm_get_state for n blocks: the engine stream packs block i into staging
// buffer i % 2 once the device-to-host copy of block i - 2 (on xstream_) has
// left it; one synchronisation at the end.
int Engine::get_states(int n, const int* blk, double* const* q) {
  if (n < 0 || (n > 0 && (!blk || !q))) return fail(FVM_ERR_INVALID, "bad block list");
  for (int i = 0; i < n; ++i) {
    if (!live_block(blk[i])) return fail(FVM_ERR_INVALID, "bad block id");
    if (!q[i]) return fail(FVM_ERR_INVALID, "null output");
  }
  if (n == 0) return FVM_OK;
  if (!laid_out_) {
    if (cap_ == 0) return fail(FVM_ERR_STATE, "no state uploaded yet");
    int rc = layout();
    if (rc) return rc;
  }
  int rc = ensure_xfer();
  if (rc) return rc;
  double* stg[2] = {d_staging_, d_staging2_};
  cudaEvent_t* copied = xev_;
  cudaEvent_t* used = xev_ + 2;
  for (int i = 0; i < n; ++i) {
    const int j = i & 1;
    const HBlock& b = blocks[blk[i]];
    const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
    if (i >= 2) CK(cudaStreamWaitEvent(stream, copied[j], 0));
    CK(launch_pack(role_[ROLE_A] + b.slab_off + b.org, cap_, (int)b.sy, (int)b.sz, (int)b.n[0], (int)b.n[1],
                   (int)b.n[2], stg[j], 0, cases[b.case_id].cfg.gamma - 1.0, stream));
    CK(cudaEventRecord(used[j], stream));
    CK(cudaStreamWaitEvent(xstream_, used[j], 0));
    CK(cudaMemcpyAsync(q[i], stg[j], bytes, cudaMemcpyDeviceToHost, xstream_));
    CK(cudaEventRecord(copied[j], xstream_));
  }
  CK(cudaEventRecord(xev_[4], xstream_));
  CK(cudaStreamWaitEvent(stream, xev_[4], 0));  // later engine work may reuse the staging buffers
  CK(cudaStreamSynchronize(xstream_));
  return FVM_OK;
}

int Engine::get_rhs(int blk, double* rhs) {
  if (!live_block(blk)) return fail(FVM_ERR_INVALID, "bad block id");
  if (!rhs) return fail(FVM_ERR_INVALID, "null output");
  const HBlock& b = blocks[blk];
  if (!cases[b.case_id].cfg.store_rhs) return fail(FVM_ERR_STATE, "store_rhs is off");
  if (!planned_ || !b.rhs_dev) return fail(FVM_ERR_STATE, "no step taken yet");
  const size_t bytes = sizeof(double) * 5 * b.n[0] * b.n[1] * b.n[2];
  CK(cudaMemcpyAsync(rhs, b.rhs_dev, bytes, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return FVM_OK;
}

int Engine::step(int nsteps) {
  if (nsteps < 0) return fail(FVM_ERR_INVALID, "nsteps < 0");
  if (!planned_) {
    if (cap_ == 0) return fail(FVM_ERR_STATE, "no state uploaded yet");
    int rc = plan();
    if (rc) return rc;
  }
  if (!prepared_) {
    int rc = prepare();
    if (rc) return rc;
  }
  CK(launch_steps(nsteps));
  return FVM_OK;
}

int Engine::read_case_state(int case_id, DevCaseState* out) {
  if (!live_case(case_id)) return fail(FVM_ERR_INVALID, "bad case id");
  // a case's device state exists from the first plan that saw it and
  // survives later re-plans
  if (!d_state_ || case_id >= state_cap_ || cases[case_id].fresh)
    return fail(FVM_ERR_STATE, "no state uploaded yet");
  CK(cudaMemcpyAsync(out, d_state_ + case_id, sizeof(DevCaseState), cudaMemcpyDeviceToHost, stream));
  int32_t err = 0;
  if (d_err_) CK(cudaMemcpyAsync(&err, d_err_, sizeof err, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (err) {
    // reported once; the context stays usable (the state of this step is not)
    CK(cudaMemsetAsync(d_err_, 0, sizeof(int32_t), stream));
    CK(cudaStreamSynchronize(stream));
    return fail(FVM_ERR_TIMEOUT, "a stage kernel's tensor copy did not arrive within 1 s");
  }
  return FVM_OK;
}

int Engine::read_all_case_states(std::vector<DevCaseState>* out) {
  out->assign(std::max(0, state_cap_), DevCaseState());
  if (!d_state_ || state_cap_ == 0) return FVM_OK;
  CK(cudaMemcpyAsync(out->data(), d_state_, sizeof(DevCaseState) * state_cap_, cudaMemcpyDeviceToHost, stream));
  int32_t err = 0;
  if (d_err_) CK(cudaMemcpyAsync(&err, d_err_, sizeof err, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (err) {
    CK(cudaMemsetAsync(d_err_, 0, sizeof(int32_t), stream));
    CK(cudaStreamSynchronize(stream));
    return fail(FVM_ERR_TIMEOUT, "a stage kernel's tensor copy did not arrive within 1 s");
  }
  return FVM_OK;
}

int Engine::time_stage(int reps, float* ms) {
  int rc = ensure_planned();
  if (rc) return rc;
  if (!prepared_) {
    rc = prepare();
    if (rc) return rc;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, stream));
  CK(launch_steps(reps));
  CK(cudaEventRecord(e1, stream));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms /= (float)std::max(1, reps);
  return FVM_OK;
}

}  // namespace fvm

// ====================================================================== C ABI
struct fvm_ctx {
  fvm::Engine eng;
  int case_id = 0;
};

// Per host thread, like the contexts: one thread's failed fvm_create never
// overwrites the message another thread is reading.
static thread_local std::string g_create_error;

// Message for fvm_last_error(NULL, ...) from entry points without a context.
void fvm_internal_set_global_error(const char* msg) { g_create_error = msg ? msg : ""; }

extern "C" {

int fvm_abi_version(void) { return FVM3D_ABI_VERSION; }

int fvm_config_default(fvm_config* c) {
  if (!c) return FVM_ERR_INVALID;
  std::memset(c, 0, sizeof *c);
  c->struct_size = (int32_t)sizeof(fvm_config);
  c->idimension = 3;
  c->equation = FVM_EQ_EULER;
  c->reconstruct = FVM_RECON_MUSCL;
  c->limiter = FVM_SCHEME_NULL;
  c->flux_split = FVM_FLUX_ROE;
  c->time_scheme = FVM_TIME_RUNGE_KUTTA;
  c->rk_stages = 3;
  c->timestep_set = FVM_DT_FIXED;
  c->compat = FVM_COMPAT_REFERENCE;
  c->precision = FVM_PREC_FP64_EXACT;
  c->store_rhs = 0;
  c->kappa = -1.0;       // ClassSpaceDiscret%kappa default (class_space_discret.f90:29)
  c->entropy_fix = 0.05; // ClassSpaceDiscret%entropy_fix_coeff (class_space_discret.f90:32)
  c->gamma = 1.4;        // ClassFlowField%gamma (class_flow_field.f90:41)
  c->dt = 0.0;
  c->cfl = 0.5;
  c->mu = 0.0;
  c->prandtl = 0.71;
  return FVM_OK;
}

int fvm_create(const fvm_config* cfg, fvm_ctx** out) {
  if (!cfg || !out) {
    g_create_error = "null argument";
    return FVM_ERR_INVALID;
  }
  *out = nullptr;
  fvm_ctx* c = new (std::nothrow) fvm_ctx();
  if (!c) return FVM_ERR_NOMEM;
  int rc = c->eng.add_case(*cfg);
  if (rc) {
    g_create_error = c->eng.err;
    delete c;
    return rc;
  }
  *out = c;
  return FVM_OK;
}

int fvm_add_block(fvm_ctx* ctx, const int64_t nvert[3], const double dr[3], int* blk) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.add_block(ctx->case_id, nvert, dr, blk);
}

int fvm_set_boundary(fvm_ctx* ctx, int blk, int region, int kind) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_boundary(blk, region, kind);
}

int fvm_connect(fvm_ctx* ctx, int blk, const int64_t range[3][2], int donor, const int64_t donor_range[3][2],
                const int32_t donor_type[3]) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.connect(blk, range, donor, donor_range, donor_type);
}

int fvm_set_state(fvm_ctx* ctx, int blk, const double* q) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_state(blk, q);
}

int fvm_get_state(fvm_ctx* ctx, int blk, double* q) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.get_state(blk, q, 0);
}

int fvm_set_states(fvm_ctx* ctx, int n, const int* blk, const double* const* q) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_states(n, blk, q);
}

int fvm_get_states(fvm_ctx* ctx, int n, const int* blk, double* const* q) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.get_states(n, blk, q);
}

int fvm_get_primitive(fvm_ctx* ctx, int blk, double* p) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.get_state(blk, p, 1);
}

int fvm_get_rhs(fvm_ctx* ctx, int blk, double* rhs) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.get_rhs(blk, rhs);
}

int fvm_step(fvm_ctx* ctx, int nsteps, double* t, double* res_abs, double* res_rel) {
  if (!ctx) return FVM_ERR_INVALID;
  int rc = ctx->eng.step(nsteps);
  if (rc) return rc;
  if (!ctx->eng.live_case(ctx->case_id)) {
    // the context's first case was removed (a batch / serving engine): no
    // outputs to report, but keep the call synchronous
    const cudaError_t e = cudaStreamSynchronize(ctx->eng.stream);
    return e == cudaSuccess ? FVM_OK : ctx->eng.cuda_fail(e, "fvm_step");
  }
  fvm::DevCaseState s;
  rc = ctx->eng.read_case_state(ctx->case_id, &s);
  if (rc) return rc;
  if (t) *t = s.t;
  if (res_abs) std::memcpy(res_abs, s.res_abs, sizeof s.res_abs);
  if (res_rel) std::memcpy(res_rel, s.res_rel, sizeof s.res_rel);
  if (s.status == FVM_ERR_NONFINITE) return ctx->eng.fail(FVM_ERR_NONFINITE, "Error: ABSRES NaN");
  if (s.status == FVM_ERR_DIVERGED)
    return ctx->eng.fail(FVM_ERR_DIVERGED, "Error: Absolute Residual Exceeds Threshold 1E10.");
  return FVM_OK;
}

int fvm_run(fvm_ctx* ctx, int64_t max_step, double total_time, double absolute_residual, double relative_residual,
            int64_t* steps_done, int* reason) {
  if (!ctx) return FVM_ERR_INVALID;
  if (absolute_residual < 0.0) return ctx->eng.fail(FVM_ERR_INVALID, "Invalid minimum absolute residual.");
  if (relative_residual < 0.0) return ctx->eng.fail(FVM_ERR_INVALID, "Invalid minimum relative residual.");
  if (total_time < -1.0E-6) return ctx->eng.fail(FVM_ERR_INVALID, "Invalid total time.");
  const double time_tol = 1.0E-10;  // class_iteration.f90 (file-local 239)
  int64_t done = 0;
  int why = FVM_STOP_NONE;
  fvm::DevCaseState s;
  std::memset(&s, 0, sizeof s);
  // a context that has stepped before starts from its current state, so the
  // stop rules see its step count, time and residuals before any new step
  if (ctx->eng.has_case_state(ctx->case_id)) {
    int rc = ctx->eng.read_case_state(ctx->case_id, &s);
    if (rc) return rc;
  }
  for (;;) {
    // converged() (class_iteration.f90, file-local 145-192); max_step counts
    // the context's steps from its first one, like the reference's iteration
    // counter, and a limit already reached stops before any step
    if (s.step != 0) {
      if (s.step >= max_step) why = FVM_STOP_MAX_STEP;
      else if (s.t > total_time - time_tol) why = FVM_STOP_MAX_TIME;
      else if (s.res_abs[5] < absolute_residual) why = FVM_STOP_ABS_RESIDUAL;
      else if (s.res_rel[5] < relative_residual) why = FVM_STOP_REL_RESIDUAL;
      else if (s.res_abs[5] > 1.0E10) {
        if (steps_done) *steps_done = done;
        return ctx->eng.fail(FVM_ERR_DIVERGED, "Error: Absolute Residual Exceeds Threshold 1E10.");
      } else if (std::isnan(s.res_abs[5])) {
        if (steps_done) *steps_done = done;
        return ctx->eng.fail(FVM_ERR_NONFINITE, "Error: ABSRES NaN");
      }
      if (why != FVM_STOP_NONE) break;
    }
    int rc = ctx->eng.step(1);
    if (rc) return rc;
    rc = ctx->eng.read_case_state(ctx->case_id, &s);
    if (rc) return rc;
    ++done;
  }
  if (steps_done) *steps_done = done;
  if (reason) *reason = why;
  return FVM_OK;
}

int fvm_get_time(fvm_ctx* ctx, double* t, double* dt, int64_t* step) {
  if (!ctx) return FVM_ERR_INVALID;
  fvm::DevCaseState s;
  std::memset(&s, 0, sizeof s);
  int rc = ctx->eng.read_case_state(ctx->case_id, &s);
  if (rc) return rc;
  if (t) *t = s.t;
  if (dt) *dt = s.dt_last;
  if (step) *step = s.step;
  return FVM_OK;
}

int fvm_last_error(const fvm_ctx* ctx, char* buf, size_t n) {
  if (!buf || n == 0) return FVM_ERR_INVALID;
  const std::string& m = ctx ? ctx->eng.err : g_create_error;
  std::snprintf(buf, n, "%s", m.c_str());
  return FVM_OK;
}

int fvm_reserve(fvm_ctx* ctx, int64_t cells) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.reserve(cells);
}

int fvm_block_cells(int idimension, const int64_t nvert[3], int64_t* cells) {
  if (!nvert || !cells || (idimension != 2 && idimension != 3)) return FVM_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (nvert[d] < 1) return FVM_ERR_INVALID;
  *cells = fvm::padded_cells(idimension, nvert);
  return FVM_OK;
}

int fvm_add_case(fvm_ctx* ctx, const fvm_config* cfg, int* case_id) {
  if (!ctx || !cfg) return FVM_ERR_INVALID;
  return ctx->eng.add_case(*cfg, case_id);
}

int fvm_add_case_block(fvm_ctx* ctx, int case_id, const int64_t nvert[3], const double dr[3], int* blk) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.add_block(case_id, nvert, dr, blk);
}

int fvm_remove_case(fvm_ctx* ctx, int case_id) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.remove_case(case_id);
}

int fvm_case_state(fvm_ctx* ctx, int case_id, double* t, double* dt, int64_t* step, double* res_abs,
                   double* res_rel, int* status) {
  if (!ctx) return FVM_ERR_INVALID;
  fvm::DevCaseState s;
  std::memset(&s, 0, sizeof s);
  int rc = ctx->eng.read_case_state(case_id, &s);
  if (rc) return rc;
  if (t) *t = s.t;
  if (dt) *dt = s.dt_last;
  if (step) *step = s.step;
  if (res_abs) std::memcpy(res_abs, s.res_abs, sizeof s.res_abs);
  if (res_rel) std::memcpy(res_rel, s.res_rel, sizeof s.res_rel);
  if (status) *status = s.status;
  return FVM_OK;
}

int fvm_tune_set(fvm_ctx* ctx, int case_id, int tile, int zchunk) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_tuning(case_id, tile, zchunk);
}

int fvm_tune_set_tail_split(fvm_ctx* ctx, int case_id, int split) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_tail_split(case_id, split);
}

int fvm_tune_time_step(fvm_ctx* ctx, int reps, float* ms_per_step) {
  if (!ctx || !ms_per_step || reps < 1) return FVM_ERR_INVALID;
  return ctx->eng.time_stage(reps, ms_per_step);
}

int fvm_profile_step(fvm_ctx* ctx, float* ms, int32_t* kinds, int cap, int* n) {
  if (!ctx || !ms || !kinds || !n || cap < 1) return FVM_ERR_INVALID;
  std::vector<int> k(cap);
  int rc = ctx->eng.profile_step(ms, k.data(), cap, n);
  for (int i = 0; i < *n; ++i) kinds[i] = k[i];
  return rc;
}

int fvm_test_drop_tensor_copies(fvm_ctx* ctx, int on) {
  if (!ctx) return FVM_ERR_INVALID;
  return ctx->eng.set_drop_copies(on != 0);
}

int fvm_test_fast_math(const double* x, int64_t n, double* rcp_out, double* rsqrt_out) {
  if (!x || !rcp_out || !rsqrt_out || n < 0) return FVM_ERR_INVALID;
  if (n == 0) return FVM_OK;
  const size_t bytes = sizeof(double) * (size_t)n;
  double* d = nullptr;
  if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) return FVM_ERR_CUDA;
  cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = fvm::launch_fast_math_probe(d, n, d + n, d + 2 * n, 0);
  if (e == cudaSuccess) e = cudaMemcpy(rcp_out, d + n, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(rsqrt_out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? FVM_OK : FVM_ERR_CUDA;
}

int fvm_kernel_launches_per_step(fvm_ctx* ctx, int* n) {
  if (!ctx || !n) return FVM_ERR_INVALID;
  int rc = ctx->eng.ensure_planned();
  if (rc) return rc;
  *n = ctx->eng.kernel_launches_per_step;
  return FVM_OK;
}

int fvm_destroy(fvm_ctx* ctx) {
  delete ctx;
  return FVM_OK;
}

}  // extern "C"
