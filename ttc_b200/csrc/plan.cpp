// Host planner: validation, index fusion, kernel choice, tile shape search, descriptor tables.
//
// Reference behaviour that is restated here (TTC, file:line inside the TTC project):
//   validation            ttc.py:733-768 (lda/ldb >= size, perm is a permutation)
//   strides from lda/ldb  CUDAtranspose.py:543-556, GPUreference.py:217-230
//                         (stride of A-dim i = prod_{k<i} lda[k], B-dim j = prod_{k<j} ldb[k])
//   index fusion          ttc_util.py:214-276 (merge A-dims i,i+1 that are also adjacent in B and
//                         unpadded); extent-1 dimensions are dropped as well, which changes no
//                         result
//   path classification   CUDAtranspose.py:34-42 (identity / perm[0]==0 / general)
// The blocking/loop-order search of GPUtransposeGenerator.py:165-285 is replaced by a cost model
// over multi-dimensional tiles (below) whose knobs the autotuner searches.
#include "plan.h"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <sstream>

int dtype_bytes(ttcb_dtype t) {
  switch (t) {
    case TTCB_S: return 4;
    case TTCB_D: return 8;
    case TTCB_C: return 8;
    case TTCB_Z: return 16;
  }
  return 0;
}

static bool dtype_complex(ttcb_dtype t) { return t == TTCB_C || t == TTCB_Z; }

static bool mul_ok(int64_t a, int64_t b, int64_t* out) { return !__builtin_mul_overflow(a, b, out); }

static int64_t gcd64(int64_t a, int64_t b) {
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// ------------------------------------------------------------------------------------------------
void fuse_problem(int rank, const int* perm, const int64_t* n, const int64_t* sA, const int64_t* sB,
                  FusedProblem& out) {
  struct Grp {
    int64_t n, sA, sB;
    int id;
    unsigned members;  // the caller's dimensions in this group (bit mask)
  };
  std::vector<Grp> a;      // groups in A order
  std::vector<int> border; // group ids in B order
  for (int i = 0; i < rank; ++i)
    if (n[i] != 1) a.push_back({n[i], sA[i], sB[i], i, 1u << i});
  for (int j = 0; j < rank; ++j)
    if (n[perm[j]] != 1) border.push_back(perm[j]);

  bool changed = true;
  while (changed) {
    changed = false;
    for (size_t k = 0; k + 1 < a.size(); ++k) {
      const Grp& g = a[k];
      const Grp& h = a[k + 1];
      size_t pg = std::find(border.begin(), border.end(), g.id) - border.begin();
      if (pg + 1 < border.size() && border[pg + 1] == h.id && h.sA == g.sA * g.n && h.sB == g.sB * g.n) {
        a[k].n *= h.n;
        a[k].members |= h.members;
        border.erase(border.begin() + pg + 1);
        a.erase(a.begin() + k + 1);
        changed = true;
        break;
      }
    }
  }
  out = FusedProblem();
  for (int i = 0; i < rank; ++i) out.fused_of[i] = -1;
  if (a.empty()) {
    out.rank = 1;
    out.perm[0] = 0;
    out.n[0] = 1;
    out.sA[0] = 1;
    out.sB[0] = 1;
    return;
  }
  out.rank = (int)a.size();
  for (int i = 0; i < out.rank; ++i)
    for (int d = 0; d < rank; ++d)
      if (a[i].members & (1u << d)) out.fused_of[d] = i;
  for (int i = 0; i < out.rank; ++i) {
    out.n[i] = a[i].n;
    out.sA[i] = a[i].sA;
    out.sB[i] = a[i].sB;
  }
  for (int j = 0; j < out.rank; ++j) {
    int id = border[j];
    for (int i = 0; i < out.rank; ++i)
      if (a[i].id == id) out.perm[j] = i;
  }
}

// ------------------------------------------------------------------------------------------------
// Cost model. Units: bytes of DRAM traffic (including wasted sector bytes) per element, plus a
// fixed per-tile overhead expressed in the same unit.
// Fixed cost of a tile (decode, barrier, pipeline step) in bytes-equivalent.
#ifndef TTCB_TILE_OVERHEAD
#define TTCB_TILE_OVERHEAD 3072.0
#endif
// Issue cost of accesses narrower than 16 bytes (per element, scaled by the missing width).
#ifndef TTCB_NARROW_COST
#define TTCB_NARROW_COST 0.6
#endif
// Efficiency factor of a run that is shorter than 128 bytes, at zero length (linear up to 1 at 128).
#ifndef TTCB_SHORT_RUN_FLOOR
#define TTCB_SHORT_RUN_FLOOR 0.75
#endif
static double run_eff(double run_bytes, int64_t align_bytes) {
  if (run_bytes <= 0) return 1e-3;
  int64_t a = std::max<int64_t>(4, std::min<int64_t>(align_bytes, 32));
  double sectors = 0;
  int cnt = 0;
  for (int64_t o = 0; o < 32; o += a) {
    sectors += std::ceil((o + run_bytes) / 32.0);
    ++cnt;
  }
  sectors /= cnt;
  double eff = run_bytes / (32.0 * sectors);
  if (run_bytes < 128) eff *= TTCB_SHORT_RUN_FLOOR + (1.0 - TTCB_SHORT_RUN_FLOOR) * run_bytes / 128.0;  // short bursts
  return eff;
}

struct TileCand {
  int64_t ext[TTCB_MAXR];  // 0 = not in tile
  int64_t P = 0;
  int64_t LA = 1, LB = 1;
  int64_t galA = 0, galB = 0;  // gcd of segment/grid offsets (elements); 0 = none
  int vecA = 1, vecB = 1;
  double cost = 1e30;
};

static void tile_orders(const FusedProblem& f, const int64_t* ext, std::vector<int>& aord, std::vector<int>& bord) {
  aord.clear();
  bord.clear();
  for (int i = 0; i < f.rank; ++i)
    if (ext[i] > 0) aord.push_back(i);
  for (int j = 0; j < f.rank; ++j)
    if (ext[f.perm[j]] > 0) bord.push_back(f.perm[j]);
}

static int64_t run_len(const std::vector<int>& order, const int64_t* ext, const int64_t* n, const int64_t* s) {
  int64_t L = 1, expect = 1;
  for (int d : order) {
    if (s[d] != expect) break;
    L *= ext[d];
    if (ext[d] < n[d]) break;
    expect = s[d] * n[d];
  }
  return L;
}

// Cost of a ragged tile relative to a complete one (per tile slot): the ragged-tile kernel checks
// every element's coordinates and moves scalars.
#ifndef TTCB_RAGGED_COST
#define TTCB_RAGGED_COST 1.5
#endif
// Cost factor of a tile that the register-offset path cannot hold (more than 1024 vectors on a
// side), which then reads its element offsets from shared-memory tables.
#ifndef TTCB_TABLE_PATH_COST
#define TTCB_TABLE_PATH_COST 1.6
#endif

static void eval_tile(const FusedProblem& f, int EA, int EB, bool beta, const ttcb_tuning& tu, TileCand& c) {
  std::vector<int> aord, bord;
  tile_orders(f, c.ext, aord, bord);
  c.P = 1;
  for (int d : aord) c.P *= c.ext[d];
  c.LA = run_len(aord, c.ext, f.n, f.sA);
  c.LB = run_len(bord, c.ext, f.n, f.sB);
  // alignment of segment starts and grid steps
  int64_t gA = 0, gB = 0;
  {
    // A: dims of the tile beyond the A run contribute to segment offsets
    int64_t acc = 1;
    bool in_run = true;
    for (int d : aord) {
      if (in_run && acc < c.LA) {
        acc *= c.ext[d];
        continue;
      }
      in_run = false;
      if (c.ext[d] > 1) gA = gcd64(gA, f.sA[d]);
    }
    acc = 1;
    in_run = true;
    for (int d : bord) {
      if (in_run && acc < c.LB) {
        acc *= c.ext[d];
        continue;
      }
      in_run = false;
      if (c.ext[d] > 1) gB = gcd64(gB, f.sB[d]);
    }
    for (int d = 0; d < f.rank; ++d) {
      int64_t e = c.ext[d] > 0 ? c.ext[d] : 1;
      if (c.ext[d] > 0 && c.ext[d] == f.n[d]) continue;  // full tile dim: no grid steps
      gA = gcd64(gA, e * f.sA[d]);
      gB = gcd64(gB, e * f.sB[d]);
    }
    gA = gcd64(gA, f.oA);
    gB = gcd64(gB, f.oB);
  }
  c.galA = gA;
  c.galB = gB;
  c.vecA = 1;
  for (int V = 16 / EA; V > 1; V /= 2)
    if (c.LA % V == 0 && (gA == 0 || gA % V == 0)) {
      c.vecA = V;
      break;
    }
  c.vecB = 1;
  for (int V = 16 / EB; V > 1; V /= 2)
    if (c.LB % V == 0 && (gB == 0 || gB % V == 0)) {
      c.vecB = V;
      break;
    }
  if (tu.vec == 1) c.vecA = c.vecB = 1;

  int64_t alA = gA == 0 ? 128 : std::min<int64_t>(128, (gA * EA) & -(gA * EA));
  int64_t alB = gB == 0 ? 128 : std::min<int64_t>(128, (gB * EB) & -(gB * EB));
  double effA = run_eff((double)c.LA * EA, alA);
  double effB = run_eff((double)c.LB * EB, alB);
  double per_elem = EA / effA + (beta ? 2.0 : 1.0) * EB / effB;
  // narrower accesses cost issue slots (the kernels are close to instruction-bound)
  per_elem += TTCB_NARROW_COST * EA * (16.0 / (c.vecA * EA) - 1.0) / 15.0 * 4.0;
  per_elem += TTCB_NARROW_COST * EB * (16.0 / (c.vecB * EB) - 1.0) / 15.0 * 4.0 * (beta ? 1.5 : 1.0);
  // the fast kernel keeps at most 4 vectors per thread and phase
  const bool fast = (c.P / c.vecA <= 1024) && (c.P / c.vecB <= 1024);
  if (!fast) per_elem *= TTCB_TABLE_PATH_COST;

  // average useful elements per tile (ragged last blocks waste a tile's fixed cost)
  double fill = 1.0;
  int64_t ntiles = 1;
  for (int d = 0; d < f.rank; ++d) {
    if (c.ext[d] == 0) {
      ntiles *= f.n[d];
    } else if (c.ext[d] < f.n[d]) {
      int64_t nb = (f.n[d] + c.ext[d] - 1) / c.ext[d];
      ntiles *= nb;
      fill *= (double)f.n[d] / (double)(nb * c.ext[d]);
    }
  }
  double tile_overhead = TTCB_TILE_OVERHEAD;  // bytes-equivalent per tile
  double cost = per_elem + tile_overhead / (c.P * fill);
  // last blocks of blocked dimensions run the element-wise ragged path
  {
    double full_frac = 1.0;
    for (int d = 0; d < f.rank; ++d)
      if (c.ext[d] > 0 && c.ext[d] < f.n[d] && f.n[d] % c.ext[d] != 0) {
        int64_t nb = (f.n[d] + c.ext[d] - 1) / c.ext[d];
        full_frac *= (double)(nb - 1) / (double)nb;
      }
    cost += (1.0 - full_frac) * per_elem * TTCB_RAGGED_COST;
  }

  // shared memory footprint and residency
  int64_t nsegA = c.P / c.LA, nsegB = c.P / c.LB;
  double smem = c.P * EA * 1.07 + 8.0 * (nsegA + nsegB) + 2.0 * c.P;
  int ctas = (int)std::min(8.0, std::floor(227.0 * 1024 / (smem + 1024)));
  if (ctas < 4) cost *= 1.0 + 0.08 * (4 - ctas);
  // too few tiles to fill 148 SMs
  double need = 148.0 * 4;
  if ((double)ntiles < need) cost *= 1.0 + 0.5 * (need - ntiles) / need;
  c.cost = cost;
}

// The run-length knob: a preference for A runs near tu.run_bytes, as a factor on the cost.
static double run_bytes_factor(const TileCand& c, int EA, const ttcb_tuning& tu) {
  if (tu.run_bytes <= 0) return 1.0;
  const double r = std::log2(std::max(1.0, (double)c.LA * EA) / tu.run_bytes);
  return 1.0 + 0.25 * std::fabs(r);
}

// Divisors of n in [8, 1024] (block sizes that leave no ragged last block), at most six of them
// spread evenly over that range on a log scale.
static void exact_blocks(int64_t n, std::vector<int64_t>& out) {
  std::vector<int64_t> all;
  for (int64_t b = 8; b <= 1024 && b < n; ++b)
    if (n % b == 0) all.push_back(b);
  out.clear();
  if (all.size() <= 6) {
    out = all;
    return;
  }
  for (int k = 0; k < 6; ++k) out.push_back(all[(all.size() - 1) * k / 5]);
}

static void block_choices(int64_t n, int64_t prefix, int EA, const std::vector<int64_t>& exact,
                          std::vector<int64_t>& out) {
  out.clear();
  out.push_back(n);
  static const int64_t base[] = {2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 24, 32, 48, 64, 96, 128, 192, 256, 512};
  for (int64_t b : base)
    if (b < n) out.push_back(b);
  for (int64_t b : exact) out.push_back(b);
  for (int64_t bytes : {128, 256, 512, 1024}) {
    int64_t b = (bytes / EA + prefix - 1) / std::max<int64_t>(prefix, 1);
    if (b >= 2 && b < n) out.push_back(b);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
}

static int64_t tile_pmax(int EA, const ttcb_tuning& tu) {
  const int64_t Pmax = tu.tile_elems > 0 ? tu.tile_elems : 16384 / EA;
  return std::min<int64_t>(Pmax, 8192);
}

// Every admissible tile shape with at most Pmax elements, in enumeration order, evaluated without
// the run-length knob (which only scales the cost).
static void enumerate_tiles(const FusedProblem& f, int EA, int EB, bool beta, int vec_knob, int64_t Pmax,
                            std::vector<TileCand>& out) {
  out.clear();
  const int r = f.rank;
  const int64_t maxseg = 1024;
  ttcb_tuning tu{};
  tu.vec = vec_knob;
  std::vector<int64_t> chA, chB;
  std::vector<std::vector<int64_t>> exact(r);
  for (int i = 0; i < r; ++i) exact_blocks(f.n[i], exact[i]);
  for (int kA = 1; kA <= r; ++kA) {
    int64_t prefA = 1;
    for (int i = 0; i < kA - 1; ++i) prefA *= f.n[i];
    if (prefA > Pmax) break;
    block_choices(f.n[kA - 1], prefA, EA, exact[kA - 1], chA);
    for (int64_t eA : chA) {
      for (int kB = 1; kB <= r; ++kB) {
        int64_t prefB = 1;
        for (int j = 0; j < kB - 1; ++j) prefB *= f.n[f.perm[j]];
        if (prefB > Pmax) break;
        block_choices(f.n[f.perm[kB - 1]], prefB, EB, exact[f.perm[kB - 1]], chB);
        for (int64_t eB : chB) {
          TileCand c;
          for (int i = 0; i < TTCB_MAXR; ++i) c.ext[i] = 0;
          bool ok = true;
          for (int i = 0; i < kA - 1; ++i) c.ext[i] = f.n[i];
          c.ext[kA - 1] = eA;
          for (int j = 0; j < kB && ok; ++j) {
            int d = f.perm[j];
            int64_t want = (j == kB - 1) ? eB : f.n[d];
            if (c.ext[d] == 0) {
              c.ext[d] = want;
            } else if (c.ext[d] != want) {
              ok = false;
            }
          }
          if (!ok) continue;
          int64_t P = 1;
          for (int i = 0; i < r; ++i)
            if (c.ext[i] > 0) {
              if (!mul_ok(P, c.ext[i], &P) || P > Pmax) {
                ok = false;
                break;
              }
            }
          if (!ok || P < 1) continue;
          int nblk = 0;
          for (int i = 0; i < r; ++i)
            if (c.ext[i] > 0 && c.ext[i] < f.n[i]) ++nblk;
          if (nblk > 2) continue;
          eval_tile(f, EA, EB, beta, tu, c);
          if (c.P / c.LA > maxseg || c.P / c.LB > maxseg) continue;
          out.push_back(c);
        }
      }
    }
  }
}

// The cheapest enumerated tile under the tuning's size limit and run-length preference (ties go to
// the longer shorter run).
static bool pick_tile(const std::vector<TileCand>& cands, int EA, const ttcb_tuning& tu, TileCand& best) {
  const int64_t Pmax = tile_pmax(EA, tu);
  bool found = false;
  for (const TileCand& c0 : cands) {
    if (c0.P > Pmax) continue;
    TileCand c = c0;
    c.cost *= run_bytes_factor(c, EA, tu);
    if (!found || c.cost < best.cost - 1e-9 ||
        (std::fabs(c.cost - best.cost) <= 1e-9 && std::min(c.LA, c.LB) > std::min(best.LA, best.LB))) {
      best = c;
      found = true;
    }
  }
  return found;
}

// Planning several tunings of one problem (the learned selector's candidates) enumerates the tile
// shapes once: while a TileEnumCache is installed on this thread, best_tile reuses its list for
// the same fused problem, types and access-width knob.
struct TileEnumCache {
  bool valid = false;
  FusedProblem f;
  int EA = 0, EB = 0, vec = 0;
  bool beta = false;
  std::vector<TileCand> cands;
};
static thread_local TileEnumCache* g_tile_cache = nullptr;

static bool same_fused(const FusedProblem& a, const FusedProblem& b) {
  if (a.rank != b.rank) return false;
  for (int i = 0; i < a.rank; ++i)
    if (a.perm[i] != b.perm[i] || a.n[i] != b.n[i] || a.sA[i] != b.sA[i] || a.sB[i] != b.sB[i]) return false;
  return true;
}

static bool best_tile(const FusedProblem& f, int EA, int EB, bool beta, const ttcb_tuning& tu, TileCand& best) {
  const int vec = tu.vec == 1 ? 1 : 0;
  if (TileEnumCache* c = g_tile_cache) {
    if (!c->valid || c->EA != EA || c->EB != EB || c->beta != beta || c->vec != vec || !same_fused(c->f, f)) {
      enumerate_tiles(f, EA, EB, beta, vec, 8192, c->cands);
      c->valid = true;
      c->f = f;
      c->EA = EA;
      c->EB = EB;
      c->beta = beta;
      c->vec = vec;
    }
    return pick_tile(c->cands, EA, tu, best);
  }
  std::vector<TileCand> cands;
  enumerate_tiles(f, EA, EB, beta, vec, tile_pmax(EA, tu), cands);
  return pick_tile(cands, EA, tu, best);
}

void plan_tile_cache_begin() {
  if (!g_tile_cache) g_tile_cache = new TileEnumCache();
  g_tile_cache->valid = false;
}

void plan_tile_cache_end() {
  delete g_tile_cache;
  g_tile_cache = nullptr;
}

// ------------------------------------------------------------------------------------------------
// Planning constants of the staged kernel's schedule: the B200's SM count and the bytes of tiles
// the whole GPU keeps in motion (see build_tile_desc).
static constexpr int kPlanSMs = 148;
static constexpr double kTargetInFlightBytes = 18.0 * 1024 * 1024;

// Ring depth S and CTAs per SM c of the staged kernel. Every resident CTA keeps S - 1 tiles in its
// ring (S - 2 of copies in flight and the one being written), so the tiles in motion on the whole
// GPU span W = c * SMs * (S - 1) * tile bytes of A and B. The planner keeps every CTA an SM holds
// (c = 0: timed over the whole 64-case 200 MiB sweep back to back, fewer CTAs per SM lost 2% with
// three and 12% with two, although single cases repeated alone ran faster with them) and picks the
// S in 3..6 whose W comes nearest 18 MiB, among the rings that let two CTAs share an SM when there
// are any: with S fixed at 3 or 4 for every case the sweep measured within 0.5% of the W rule, and for
// single cases rings far from it lost 5-15%. Problems too small to
// fill the GPU twice keep the earlier rule (four stages while four CTAs fit, else three).
// smem_for(S) is the dynamic shared memory of an S-stage ring; fixed_S (3..kMaxStages, else 0) is a
// schedule's explicit ring depth.
struct StageChoice {
  int S = 3;
  int c = 0;
};

template <typename SmemFn>
static StageChoice choose_stages(int64_t P, int EA, int EB, bool beta, int vecA, int vecB, int64_t nfull,
                                 const SmemFn& smem_for, int fixed_S) {
  StageChoice out;
  out.S = smem_for(4) <= 56 * 1024 ? 4 : 3;
  const bool fixed = fixed_S >= 3 && fixed_S <= ttcb::kMaxStages;
  const int64_t tile_bytes = P * (int64_t)(EA + EB * (beta ? 2 : 1));
  const int reg_ctas = ttcb::async_min_blocks(vecA * EA, vecB * EB, beta);
  // rings that leave room for a second CTA on each SM come first: with one CTA per SM the SM idles
  // at every tile barrier (the 1000x768x16 fp32 beta = 1 transposition ran at 4.4 TB/s with four
  // stages and one CTA per SM, at 5.4 TB/s with three stages and two)
  double best = 1e30;
  int bS = 0, bc = 0;
  for (int S = 3; S <= 6; ++S) {
    if (fixed && S != fixed_S) continue;
    if (smem_for(S) > 200 * 1024) continue;
    const int64_t per_cta = smem_for(S) + (int64_t)ttcb::kAsyncStaticSmem + 1024;
    const int cmax = (int)std::min<int64_t>(reg_ctas, (227 * 1024) / per_cta);
    if (cmax < 1) continue;
    const double W = (double)cmax * kPlanSMs * (S - 1) * (double)tile_bytes;
    const double key = std::fabs(std::log(W / kTargetInFlightBytes));
    const bool better = bS == 0 || (std::min(cmax, 2) > std::min(bc, 2)) ||
                        (std::min(cmax, 2) == std::min(bc, 2) && key < best - 1e-9);
    if (better) {
      best = key;
      bS = S;
      bc = cmax;
    }
  }
  if (bS && nfull >= 2LL * 4 * kPlanSMs) out.S = bS;
  if (fixed) out.S = fixed_S;
  return out;
}

// Shifted A runs (TileDesc::shiftA) for a tile whose A runs 16-byte accesses cannot reach directly
// but that are at least two 16-byte chunks long, on the staged kernel only, when the schedule asks
// for them: over the 200 MiB sweep they made 3 of the 19 cases they apply to faster (by 3-8%) and
// the others 1-13% slower, so the planner leaves them to the search.
static bool wants_shifted_runs(const TileCand& c, int EA, const ttcb_tuning& tu) {
  const int VM = 16 / EA;
  return EA < 16 && c.vecA < VM && c.LA >= 2 * VM && tu.vec != 1 && tu.shifted_runs == 1 &&
         (tu.tile_variant == 0 || tu.tile_variant == 3);
}

// Bulk A copies (TileDesc::bulkA): possible on the staged kernel when 16-byte vectors reach every A
// run, or the runs are shifted; used when the schedule asks for them (bulk_copies = 1). Timed over
// the 200 MiB sweep back to back with round-robin tiles, copies of 320 bytes and more were up to 22%
// faster than per-thread copies (mean +5%) and shorter ones 16-86% slower (a bulk copy costs the copy
// unit about as much as a short run gains); with the planner's claimed tiles their effect ranged
// from -21% to +11% per case with no rule in the run length, beta or tile size that separates the
// two, and the sweep as a whole was 0.7% slower. So the planner leaves them to the search.
static bool bulk_possible(const TileCand& c, int EA, const ttcb_tuning& tu, bool shift) {
  return tu.bulk_copies == 1 && tu.vec != 1 && (tu.tile_variant == 0 || tu.tile_variant == 3) &&
         (shift || c.vecA * EA == 16);
}

static void build_tile_desc(ttcb_plan* p, const TileCand& c, int EA) {
  const FusedProblem& f = p->f;
  const int EB_ = dtype_bytes(p->tb);
  std::vector<int> aord, bord;
  tile_orders(f, c.ext, aord, bord);
  // tile strides in A order / B order
  int64_t tsA[TTCB_MAXR] = {0}, tsB[TTCB_MAXR] = {0};
  {
    int64_t acc = 1;
    for (int d : aord) {
      tsA[d] = acc;
      acc *= c.ext[d];
    }
    acc = 1;
    for (int d : bord) {
      tsB[d] = acc;
      acc *= c.ext[d];
    }
  }
  const int64_t P = c.P;
  // padding of the shared-memory slots: consecutive p (A run) are sigma apart in q
  int pshift = 30, pad = 0;
  {
    int64_t sigma = tsB[aord[0]];
    if (sigma >= 4) {
      int k = __builtin_ctzll((unsigned long long)sigma);
      if (k >= 2) {
        pshift = std::min(k, 12);
        pad = 1;
      }
    }
  }
  auto phys = [&](int64_t q) { return q + (pad ? (q >> pshift) : 0); };
  int64_t phys_size = phys(P - 1) + 1;

  int64_t nsegA = P / c.LA, nsegB = P / c.LB;
  std::vector<int64_t> segA(nsegA), segB(nsegB);
  std::vector<uint16_t> ptab(P);
  std::vector<int64_t> p_of_q(P);
  for (int64_t pp = 0; pp < P; ++pp) {
    int64_t rem = pp, offA = 0, q = 0;
    for (int d : aord) {
      int64_t cd = rem % c.ext[d];
      rem /= c.ext[d];
      offA += cd * f.sA[d];
      q += cd * tsB[d];
    }
    ptab[pp] = (uint16_t)phys(q);
    p_of_q[q] = pp;
    if (pp % c.LA == 0) segA[pp / c.LA] = offA;
  }
  // Staged layout of the asynchronous-copy kernel: element p at p + (p / sigma) * padA. sigma (a
  // multiple of the A vector that divides into whole vectors) and padA (a multiple of the A vector)
  // are the pair that minimises shared-memory bank conflicts of the store-phase gather, replayed on
  // the host for the first warps (32 lanes, 4-byte banks).
  const int EAw = EA >= 4 ? EA / 4 : 1;
  int64_t sigma = c.LA;
  auto staged = [&](int64_t pp, int64_t padA) { return pp + (pp / sigma) * padA; };
  // Shifted A runs: when 16-byte accesses cannot reach A's runs directly (their length or offsets
  // are not multiples of V = 16 / EA elements) but the runs are at least 2V long, each run is copied
  // as the 16-byte chunks that cover it (see TileDesc::shiftA): up to LA / V + 2 copies instead of LA
  // (fp32) or LA / 2 (fp64) narrow ones. Run s then sits at s * shiftW + (segA[s] mod V).
  const int VM = 16 / EA;
  const bool shift = wants_shifted_runs(c, EA, p->tuning);
  // bulk copies of plain runs need padding points that split runs into equal pieces (sigma a
  // multiple or a divisor of LA); decided below with the layout
  bool bulk = bulk_possible(c, EA, p->tuning, shift);
  const int64_t CM = shift ? (2 * VM - 3 + c.LA) / VM + 1 : 0;  // chunk slots per run
  int64_t shiftW = CM * VM;
  auto staged_shift = [&](int64_t pp, int64_t W) {
    const int64_t s = pp / c.LA;
    return s * W + (((segA[s] % VM) + VM) % VM) + (pp - s * c.LA);
  };
  // The register path's lane map (TileDesc::map_log2s): with map_s > 0 a warp takes map_s B vectors
  // from each of 32 / map_s consecutive B runs; vec_of gives the B vector of thread slot i.
  const int64_t map_nx = c.LB / c.vecB, map_ny = P / c.LB;
  int map_s = 0;
  bool map_sorted = false;
  // the B runs in the order of the A position of their first element (stable)
  std::vector<int64_t> run_order(map_ny);
  for (int64_t y = 0; y < map_ny; ++y) run_order[y] = y;
  std::stable_sort(run_order.begin(), run_order.end(),
                   [&](int64_t a, int64_t b) { return p_of_q[a * c.LB] < p_of_q[b * c.LB]; });
  // -1: a slot past the tile's B runs
  auto vec_of = [&](int64_t i) -> int64_t {
    if (!map_s) return i * c.vecB < P ? i : -1;
    const int64_t w = i >> 5, l = i & 31, nbx = map_nx / map_s;
    const int64_t y = (w / nbx) * (32 / map_s) + l / map_s;
    if (y >= map_ny) return -1;
    return (w % nbx) * map_s + (l % map_s) + map_nx * (map_sorted ? run_order[y] : y);
  };
  auto map_slots = [&](int ms) -> int64_t {
    const int64_t rows = 32 / ms;
    return (map_nx / ms) * ((map_ny + rows - 1) / rows) * 32;
  };
  // A warp's 8-byte loads are served per half-warp and its 16-byte loads per quarter-warp, so the
  // wavefronts of one load are the sum over those lane groups of the busiest bank's count. The cost
  // is the wavefronts beyond one per lane group (0 = no conflicts), over the first four warps.
  const int group = 32 / EAw;
  auto gather_cost = [&](int64_t padA) {
    int64_t cost = 0;
    const int vb = c.vecB;
    for (int w = 0; w < 4; ++w) {
      for (int j = 0; j < vb; ++j) {
        for (int g0 = 0; g0 < 32; g0 += group) {
          int cnt[32] = {0};
          int mx = 0;
          for (int lane = g0; lane < g0 + group; ++lane) {
            const int64_t v = vec_of((int64_t)w * 32 + lane);
            if (v < 0) continue;
            int64_t word = (shift ? staged_shift(p_of_q[v * vb + j], shiftW + padA)
                                  : staged(p_of_q[v * vb + j], padA)) * EAw;
            for (int x = 0; x < EAw; ++x) {
              int b = (int)((word + x) & 31);
              mx = std::max(mx, ++cnt[b]);
            }
          }
          cost += mx > 0 ? mx - 1 : 0;
        }
      }
    }
    return cost;
  };
  int64_t padA = 0;
  {
    // periods: the A run, small multiples of the A-order stride of each tile dimension, and every
    // multiple of the A vector up to 64 elements
    std::vector<int64_t> sigmas = {c.LA};
    for (int d : aord)
      for (int64_t m = 1; m <= 8; m *= 2)
        if (tsA[d] > 1 && m * tsA[d] < P && (m * tsA[d]) % c.vecA == 0) sigmas.push_back(m * tsA[d]);
    for (int64_t k = c.vecA; k <= 64 && k < P; k += c.vecA) sigmas.push_back(k);
    // one wavefront per lane group and load is the floor; stop searching once it is reached
    const int64_t ideal = 0;
    int64_t best_cost = -1, best_sigma = c.LA, best_pad = 0;
    if (shift) {
      // the run stride: the chunk slots plus 0..8 chunks of padding, the fewest conflicts
      for (int k = 0; k <= 8; ++k) {
        const int64_t cand = (int64_t)k * VM;
        if ((P / c.LA) * (shiftW + cand) > 65535) break;
        const int64_t cc = gather_cost(cand);
        if (best_cost < 0 || cc < best_cost) {
          best_cost = cc;
          best_pad = cand;
        }
        if (best_cost == ideal) break;
      }
      shiftW += best_pad;
    }
    // the (period, pad) pair with the fewest conflicts; with min_piece > 0 only periods that cut the
    // runs into equal pieces of at least min_piece elements (bulk copies)
    auto search = [&](int64_t min_piece, int64_t& out_cost, int64_t& out_sigma, int64_t& out_pad) {
      out_cost = -1;
      out_sigma = c.LA;
      out_pad = 0;
      for (int64_t sg : sigmas) {
        if (out_cost == ideal) break;
        if (min_piece > 0 && ((sg % c.LA != 0 && c.LA % sg != 0) || std::min<int64_t>(sg, c.LA) < min_piece)) continue;
        sigma = sg;
        for (int k = 0; k <= 8; ++k) {
          const int64_t cand = (int64_t)k * c.vecA;
          if (k && (cand > 32 || cand > sg)) break;
          if ((P - 1) / sg * cand + P > 65535) continue;
          const int64_t cc = gather_cost(cand);
          if (out_cost < 0 || cc < out_cost) {
            out_cost = cc;
            out_sigma = sg;
            out_pad = cand;
          }
          if (out_cost == ideal) break;
        }
      }
    };
    if (!shift) {
      search(0, best_cost, best_sigma, best_pad);
      if (bulk) {
        // the fewest conflicts among the periods that cut runs into whole 16-byte pieces
        int64_t bc = -1, bs = c.LA, bp = 0;
        search(1, bc, bs, bp);
        if (bc >= 0) {
          best_cost = bc;
          best_sigma = bs;
          best_pad = bp;
        } else {
          bulk = false;
        }
      }
      // Lane maps (schedule lane_map = 1), when the layout alone leaves conflicts and the tile can
      // take the register path (every thread's B vectors in registers): the pads are multiples of
      // the A vector, so lanes whose A positions differ by multiples of a larger power of two meet
      // in the same banks whatever the layout; lanes spread over several B runs read different A
      // positions. Each lane group keeps at least one whole 32-byte sector of its B run. Timed over
      // the 200 MiB sweep back to back, maps on the 21 cases the model picked them for were up to
      // 18% slower and at most 1.4% faster (a warp's stores then reach 2 to 16 B runs instead of one
      // or two): the gather's conflicts are not what limits those cases, so maps stay opt-in.
      const bool reg_shape = P / c.vecA <= 4 * ttcb::kThreads && P / c.vecB <= 4 * ttcb::kThreads &&
                             P * EB_ < 65536 && p->tuning.lane_map == 1;
      if (best_cost > ideal && reg_shape) {
        int best_map = 0;
        bool best_sorted = false;
        for (int ms = 1; ms <= 16 && best_cost > ideal; ms *= 2) {
          if ((int64_t)ms * c.vecB * EB_ < 32 || map_nx % ms != 0 || map_slots(ms) > 4 * ttcb::kThreads) continue;
          for (int so = 0; so < 2 && best_cost > ideal; ++so) {
            map_s = ms;
            map_sorted = so == 1;
            int64_t mc = -1, msg = c.LA, mp = 0;
            search(bulk ? 1 : 0, mc, msg, mp);
            if (mc >= 0 && mc < best_cost) {
              best_cost = mc;
              best_sigma = msg;
              best_pad = mp;
              best_map = ms;
              best_sorted = map_sorted;
            }
          }
        }
        map_s = best_map;
        map_sorted = best_sorted;
      }
    }
    sigma = shift ? c.LA : best_sigma;
    padA = shift ? 0 : best_pad;
  }
  const int64_t bulk_pieces = (bulk && !shift && sigma < c.LA) ? c.LA / sigma : 1;
  const int64_t staged_size = shift ? (P / c.LA) * shiftW : staged(P - 1, padA) + 1;
  std::vector<uint16_t> gtab(P);
  for (int64_t q = 0; q < P; ++q)
    gtab[q] = (uint16_t)(shift ? staged_shift(p_of_q[q], shiftW) : staged(p_of_q[q], padA));
  for (int64_t s = 0; s < nsegB; ++s) {
    int64_t rem = s * c.LB, offB = 0;
    for (int d : bord) {
      int64_t cd = rem % c.ext[d];
      rem /= c.ext[d];
      offB += cd * f.sB[d];
    }
    segB[s] = offB;
  }

  TileDesc td;
  std::memset(&td, 0, sizeof(td));
  td.shiftA = shift ? 1 : 0;
  td.shiftW = (int32_t)(shift ? shiftW : 0);
  td.shiftCM = (int32_t)CM;
  td.bulkA = bulk ? 1 : 0;
  td.bulk_pieces = (int32_t)bulk_pieces;
  td.map_log2s = map_s ? __builtin_ctz((unsigned)map_s) : -1;
  td.map_nx = (int32_t)(map_s ? map_nx : 0);
  td.map_nbx = (int32_t)(map_s ? map_nx / map_s : 0);
  td.map_vb = map_s ? c.vecB : 0;
  td.map_ny = (int32_t)(map_s ? map_ny : 0);
  td.map_nslots = (int32_t)(map_s ? map_slots(map_s) : 0);
  td.divPieces = make_fastdiv((uint32_t)bulk_pieces);
  td.divCM = make_fastdiv((uint32_t)std::max<int64_t>(CM, 1));
  td.P = (int32_t)P;
  td.LA = (int32_t)c.LA;
  td.LB = (int32_t)c.LB;
  td.nsegA = (int32_t)nsegA;
  td.nsegB = (int32_t)nsegB;
  td.pshift = pshift;
  td.pad = pad;
  td.phys_size = (int32_t)phys_size;
  td.divLA = make_fastdiv((uint32_t)c.LA);
  td.divLB = make_fastdiv((uint32_t)c.LB);

  // grid dimensions, fastest first, in the requested loop order
  std::vector<int> gdims;
  if (p->loop_order == 1) {
    for (int j = 0; j < f.rank; ++j) gdims.push_back(f.perm[j]);
  } else if (p->loop_order == 2) {
    for (int i = f.rank - 1; i >= 0; --i) gdims.push_back(i);
  } else if (p->loop_order == 4) {
    // the caller's loop order: each fused dimension at the first appearance of one of its members
    int order[TTCB_MAXR];
    unpack_raster(p->tuning, p->rank, order);
    bool seen[TTCB_MAXR] = {false};
    for (int k = 0; k < p->rank; ++k) {
      const int fd = f.fused_of[order[k]];
      if (fd >= 0 && !seen[fd]) {
        seen[fd] = true;
        gdims.push_back(fd);
      }
    }
  } else {
    for (int i = 0; i < f.rank; ++i) gdims.push_back(i);
  }
  int ng = 0, nb = 0;
  int64_t ntiles = 1;
  int gdim_of[TTCB_MAXR];  // fused dimension of each grid dimension
  for (int d : gdims) {
    if (c.ext[d] > 0 && c.ext[d] == f.n[d]) continue;
    int64_t e = c.ext[d] > 0 ? c.ext[d] : 1;
    int64_t cnt = (f.n[d] + e - 1) / e;
    gdim_of[ng] = d;
    GridDimDesc& g = td.g[ng++];
    g.div = make_fastdiv((uint32_t)cnt);
    g.divf = make_fastdiv((uint32_t)(c.ext[d] > 0 && f.n[d] % e != 0 ? cnt - 1 : cnt));
    g.strideA = e * f.sA[d];
    g.strideB = e * f.sB[d];
    g.n = f.n[d];
    g.e = (int32_t)e;
    g.blocked = -1;
    if (c.ext[d] > 0) {
      g.blocked = nb;
      BlockedDesc& b = td.bd[nb++];
      b.tsA = make_fastdiv((uint32_t)tsA[d]);
      b.tsB = make_fastdiv((uint32_t)tsB[d]);
      b.ext = make_fastdiv((uint32_t)e);
    }
    ntiles *= cnt;
  }
  td.ngrid = ng;
  td.nblocked = nb;
  p->nraster = ng;
  for (int k = 0; k < ng; ++k) p->raster[k] = gdim_of[k];
  td.ntiles = (int32_t)ntiles;
  td.rag_a = td.rag_b = -1;
  for (int k = 0; k < ng; ++k)
    if (td.g[k].blocked >= 0 && td.g[k].n % td.g[k].e != 0) {
      if (td.rag_a < 0)
        td.rag_a = k;
      else
        td.rag_b = k;
    }
  p->rag_dim[0] = p->rag_dim[1] = -1;
  p->rag_start[0] = p->rag_start[1] = 0;
  for (int k = 0; k < 2; ++k) {
    const int gk = k == 0 ? td.rag_a : td.rag_b;
    if (gk < 0) continue;
    p->rag_dim[k] = gdim_of[gk];
    p->rag_start[k] = (int64_t)(td.g[gk].div.d - 1) * td.g[gk].e;
  }
  {
    const int64_t ca = td.rag_a >= 0 ? td.g[td.rag_a].div.d : 1, cb = td.rag_b >= 0 ? td.g[td.rag_b].div.d : 1;
    td.nrag0 = td.rag_a >= 0 ? (int32_t)(ntiles / ca) : 0;
    td.nrag1 = td.rag_b >= 0 ? (int32_t)(ntiles / ca / cb * (ca - 1)) : 0;
    int64_t nfull = 1;
    for (int k = 0; k < ng; ++k) nfull *= td.g[k].divf.d;
    td.nfull = (int32_t)nfull;
  }

  auto al16 = [](int64_t x) { return (x + 15) & ~int64_t(15); };
  int64_t off = al16(sizeof(TileDesc));
  td.off_segA = (int32_t)off;
  off = al16(off + 8 * nsegA);
  td.off_segB = (int32_t)off;
  off = al16(off + 8 * nsegB);
  td.off_perm = (int32_t)off;
  off = al16(off + 2 * P);
  td.off_gtab = (int32_t)off;
  off = al16(off + 2 * P);
  td.off_runs = 0;
  if (map_s && map_sorted) {
    td.off_runs = (int32_t)off;
    off = al16(off + 2 * map_ny);
  }
  int64_t smem = al16(phys_size * EA) + 8 * nsegA + 8 * nsegB + al16(2 * P);
  td.smem_bytes = (int32_t)smem;
  {
    // the fast kernel keeps tile-relative offsets in 32-bit registers
    int64_t mA = 0, mB = 0;
    for (int64_t x : segA) mA = std::max(mA, x + c.LA);
    for (int64_t x : segB) mB = std::max(mB, x + c.LB);
    td.fast = (mA < (int64_t(1) << 31) && mB < (int64_t(1) << 31) && P / c.vecA <= 1024 && P / c.vecB <= 1024) ? 1 : 0;
    td.padA = (int32_t)padA;
    td.sigmaA = (int32_t)sigma;
    td.divSigmaA = make_fastdiv((uint32_t)sigma);
    td.stage_elems = (int32_t)std::max<int64_t>(staged_size, phys_size);
    const bool beta = p->beta_nonzero != 0;
    const int EB = dtype_bytes(p->tb);
    auto smem_for = [&](int S) {
      return (int64_t)ttcb::async_smem_bytes(S, td.stage_elems, (int)P, (int)nsegA, (int)nsegB, EA, EB, beta);
    };
    {
      const StageChoice sc = choose_stages(P, EA, dtype_bytes(p->tb), beta, shift ? VM : c.vecA, c.vecB, td.nfull, smem_for,
                                           p->tuning.stages);
      td.nstages = sc.S;
      p->ctas_per_sm = p->tuning.ctas_per_sm > 0 ? p->tuning.ctas_per_sm : sc.c;
    }
    if (p->tuning.stages >= 3 && p->tuning.stages <= ttcb::kMaxStages) td.nstages = p->tuning.stages;
    td.async_ok = (mA < (int64_t(1) << 31) && mB < (int64_t(1) << 31) && td.stage_elems < 65536 &&
                   smem_for(td.nstages) <= 200 * 1024) ? 1 : 0;
    p->smem_async = (int)smem_for(td.nstages);
    td.reg_ok = (td.fast && td.stage_elems * (int64_t)EA < 65536 && P * (int64_t)EB < 65536) ? 1 : 0;
    // with shifted runs every chunk slot is a copy: the register path holds four per thread (bulk
    // copies of shifted runs hold none)
    if (shift && !bulk && (P / c.LA) * CM > 4 * 256) td.reg_ok = 0;
    // the staged kernel leaves ragged tiles to the ragged-tile kernel, whose tables must fit too
    if (td.nrag0 + td.nrag1 > 0 && ttcb::ragged_smem_bytes((int)phys_size, EA, (int)P) > 200 * 1024) td.async_ok = 0;
  }

  p->host_desc.assign(off, 0);
  std::memcpy(p->host_desc.data(), &td, sizeof(td));
  std::memcpy(p->host_desc.data() + td.off_segA, segA.data(), 8 * nsegA);
  std::memcpy(p->host_desc.data() + td.off_segB, segB.data(), 8 * nsegB);
  std::memcpy(p->host_desc.data() + td.off_perm, ptab.data(), 2 * P);
  std::memcpy(p->host_desc.data() + td.off_gtab, gtab.data(), 2 * P);
  if (td.off_runs)
    for (int64_t y = 0; y < map_ny; ++y) {
      const uint16_t r = (uint16_t)run_order[y];
      std::memcpy(p->host_desc.data() + td.off_runs + 2 * y, &r, 2);
    }
  p->smem_bytes = (int)smem;
  p->smem_fast = (int)al16(phys_size * EA);
  p->smem_ragged = (int)ttcb::ragged_smem_bytes((int)phys_size, EA, (int)P);
  p->vecA = shift ? VM : c.vecA;  // shifted runs copy 16-byte chunks
  p->vecB = c.vecB;
  p->est_cost = c.cost;
}

static ttcb_status build_row_desc(ttcb_plan* p, std::string& err) {
  const FusedProblem& f = p->f;
  const int EA = dtype_bytes(p->ta), EB = dtype_bytes(p->tb);
  RowDesc rd;
  std::memset(&rd, 0, sizeof(rd));
  rd.w = f.n[0];
  int64_t g = 0;
  for (int i = 1; i < f.rank; ++i) {
    g = gcd64(g, f.sA[i]);
    g = gcd64(g, f.sB[i]);
  }
  g = gcd64(gcd64(g, f.oA), f.oB);
  int V = 16 / std::max(EA, EB);
  while (V > 1 && !(g == 0 || g % V == 0)) V /= 2;
  if (p->tuning.vec == 1) V = 1;
  const int64_t chunk_max = 32 * V * 8;
  int64_t chunk = rd.w <= chunk_max ? rd.w : chunk_max;
  int64_t nchunk = (rd.w + chunk - 1) / chunk;
  int64_t rows = 1;
  rd.nd = f.rank - 1;
  for (int i = 1; i < f.rank; ++i) {
    rows *= f.n[i];
    rd.div[i - 1] = make_fastdiv((uint32_t)f.n[i]);
    rd.sA[i - 1] = f.sA[i];
    rd.sB[i - 1] = f.sB[i];
    if (f.n[i] >= (int64_t(1) << 31)) {
      err = "row dimension extent >= 2^31 is not supported";
      return TTCB_ERR_UNSUPPORTED;
    }
  }
  int64_t units = rows * nchunk;
  if (units >= (int64_t(1) << 31) || nchunk >= (int64_t(1) << 31)) {
    err = "row copy: more than 2^31 work units";
    return TTCB_ERR_UNSUPPORTED;
  }
  rd.chunk = (int32_t)chunk;
  rd.nchunk = (int32_t)nchunk;
  rd.nunits = (int32_t)units;
  rd.divChunk = make_fastdiv((uint32_t)nchunk);
  p->host_desc.assign(sizeof(RowDesc), 0);
  std::memcpy(p->host_desc.data(), &rd, sizeof(rd));
  p->smem_bytes = 0;
  p->vecA = p->vecB = V;
  double eff = run_eff((double)rd.w * std::max(EA, EB), (g == 0 ? 128 : std::min<int64_t>(128, (g * EA) & -(g * EA))));
  p->est_cost = (EA + (p->beta_nonzero ? 2.0 : 1.0) * EB) / eff;
  return TTCB_OK;
}

bool unpack_raster(const ttcb_tuning& tu, int rank, int* order) {
  bool seen[TTCB_MAXR] = {false};
  for (int k = 0; k < rank; ++k) {
    const uint32_t w = (uint32_t)(k < 8 ? tu.raster_lo : tu.raster_hi);
    const int d = (int)((w >> (4 * (k % 8))) & 0xfu) - 1;
    if (d < 0 || d >= rank || seen[d]) return false;
    seen[d] = true;
    order[k] = d;
  }
  // nothing may follow the last dimension
  for (int k = rank; k < 10; ++k) {
    const uint32_t w = (uint32_t)(k < 8 ? tu.raster_lo : tu.raster_hi);
    if ((w >> (4 * (k % 8))) & 0xfu) return false;
  }
  return true;
}

// ------------------------------------------------------------------------------------------------
ttcb_status plan_build_host(ttcb_plan* p, std::string& err) {
  const int r = p->rank;
  if (r < 1 || r > TTCB_MAXR) {
    err = "rank must be in [1, " + std::to_string(TTCB_MAXR) + "], got " + std::to_string(r);
    return TTCB_ERR_RANK;
  }
  {
    bool seen[TTCB_MAXR] = {false};
    for (int j = 0; j < r; ++j) {
      int d = p->perm[j];
      if (d < 0 || d >= r || seen[d]) {
        err = "permutation is invalid";
        return TTCB_ERR_BAD_PERM;
      }
      seen[d] = true;
    }
  }
  for (int i = 0; i < r; ++i) {
    if (p->size[i] < 0) {
      err = "size[" + std::to_string(i) + "] is negative";
      return TTCB_ERR_INVALID_ARG;
    }
    if (p->lda[i] < p->size[i]) {
      err = "the leading dimension of A for dim " + std::to_string(i) + " is smaller than allowed (it must be >= " +
            std::to_string(p->size[i]) + ")";
      return TTCB_ERR_BAD_LD;
    }
  }
  for (int j = 0; j < r; ++j) {
    if (p->ldb[j] < p->size[p->perm[j]]) {
      err = "the leading dimension of B for dim " + std::to_string(j) + " is smaller than allowed (it must be >= " +
            std::to_string(p->size[p->perm[j]]) + ")";
      return TTCB_ERR_BAD_LD;
    }
  }
  if ((int)p->ta < 0 || (int)p->ta > 3 || (int)p->tb < 0 || (int)p->tb > 3 ||
      dtype_complex(p->ta) != dtype_complex(p->tb)) {
    err = "unsupported data type pair (valid: s, d, c, z, sd, ds, cz, zc)";
    return TTCB_ERR_DTYPE;
  }
  const int EA = dtype_bytes(p->ta), EB = dtype_bytes(p->tb);

  // strides
  int64_t sA[TTCB_MAXR], sB[TTCB_MAXR], sBpos[TTCB_MAXR];
  sA[0] = 1;
  sBpos[0] = 1;
  for (int i = 1; i < r; ++i) {
    if (!mul_ok(sA[i - 1], std::max<int64_t>(p->lda[i - 1], 1), &sA[i]) ||
        !mul_ok(sBpos[i - 1], std::max<int64_t>(p->ldb[i - 1], 1), &sBpos[i])) {
      err = "stride overflow";
      return TTCB_ERR_UNSUPPORTED;
    }
  }
  for (int j = 0; j < r; ++j) sB[p->perm[j]] = sBpos[j];
  int64_t N = 1;
  for (int i = 0; i < r; ++i) {
    if (!mul_ok(N, p->size[i], &N)) {
      err = "element count overflow";
      return TTCB_ERR_UNSUPPORTED;
    }
  }
  p->N = N;
  p->empty = (N == 0);
  p->streaming = (p->tuning.streaming == 1) || (p->tuning.streaming == 0 && !p->beta_nonzero);
  if (p->beta_nonzero) p->streaming = false;
  p->loop_order = p->tuning.loop_order ? p->tuning.loop_order : 3;  // the tile planner may choose
  if (p->tuning.loop_order < 0 || p->tuning.loop_order > 4) {
    err = "loop_order must be in [0, 4]";
    return TTCB_ERR_INVALID_ARG;
  }
  if (p->tuning.loop_order == 4) {
    int order[TTCB_MAXR];
    if (!unpack_raster(p->tuning, r, order)) {
      err = "the loop order (raster_lo/raster_hi) is not a permutation of the dimensions";
      return TTCB_ERR_BAD_PERM;
    }
  }
  if (p->empty) {
    p->kernel = 0;
    p->f.rank = 0;
    return TTCB_OK;
  }
  fuse_problem(r, p->perm, p->size, sA, sB, p->f);
  p->f.oA = p->base_offA;
  p->f.oB = p->base_offB;
  const FusedProblem& f = p->f;
  for (int i = 0; i < f.rank; ++i)
    if (f.n[i] >= (int64_t(1) << 31) && !(f.perm[0] == 0 && i == 0)) {
      err = "a fused extent >= 2^31 outside the shared stride-1 dimension is not supported";
      return TTCB_ERR_UNSUPPORTED;
    }

  const bool beta = p->beta_nonzero != 0;
  // kernel choice
  bool row_possible = (f.perm[0] == 0 && f.sA[0] == 1 && f.sB[0] == 1);
  TileCand best;
  bool have_tile = false;
  if (!(row_possible && f.n[0] >= (int64_t(1) << 31))) have_tile = best_tile(f, EA, EB, beta, p->tuning, best);
  int kernel = 0;
  if (p->tuning.kernel == TTCB_KERNEL_ROW) {
    if (!row_possible) {
      err = "row kernel requested but A and B do not share their stride-1 dimension";
      return TTCB_ERR_UNSUPPORTED;
    }
    kernel = TTCB_KERNEL_ROW;
  } else if (p->tuning.kernel == TTCB_KERNEL_TILE) {
    if (!have_tile) {
      err = "no tile shape fits this problem";
      return TTCB_ERR_UNSUPPORTED;
    }
    kernel = TTCB_KERNEL_TILE;
  } else {
    if (row_possible) {
      double rb = (double)f.n[0] * std::max(EA, EB);
      double row_cost = (EA + (beta ? 2.0 : 1.0) * EB) / run_eff(rb, 16);
      // short shared rows are slow to copy one warp per row; the tile kernel packs many of them
      // (measured on 200 MiB cases: rows of 624 bytes 3846 GB/s by row, 4985 by tile; rows of
      // 2-3 KB 5150-5450 by row, 4850-5250 by tile)
      (void)row_cost;
      kernel = (!have_tile || rb >= 1024) ? TTCB_KERNEL_ROW : TTCB_KERNEL_TILE;
    } else {
      if (!have_tile) {
        err = "no tile shape fits this problem";
        return TTCB_ERR_UNSUPPORTED;
      }
      kernel = TTCB_KERNEL_TILE;
    }
  }
  p->kernel = kernel;
  if (kernel == TTCB_KERNEL_ROW) return build_row_desc(p, err);
  int64_t ntiles = 1;
  {
    // tile counts must fit the kernels' 32-bit tile index
    for (int d = 0; d < f.rank; ++d) {
      int64_t e = best.ext[d] > 0 ? best.ext[d] : 1;
      if (best.ext[d] > 0 && best.ext[d] == f.n[d]) continue;
      ntiles *= (f.n[d] + e - 1) / e;
      if (ntiles >= (int64_t(1) << 31)) {
        err = "more than 2^31 tiles";
        return TTCB_ERR_UNSUPPORTED;
      }
    }
  }
  // Raster of the tile grid when the schedule leaves it to the planner: B-major when B's runs are
  // shorter than 256 bytes and B exceeds 64 MiB (half of L2), else A-major. Short B runs leave
  // partially written sectors at the run ends; the B-major raster writes the tiles that share them
  // together, while the sectors are still in L2, instead of a pass apart (measured on 2000 timed
  // problems: 8% faster on the 138 this rule selects, 79% of them faster).
  if (p->tuning.loop_order == 0)
    p->loop_order = (best.LB * EB < 256 && p->N * (int64_t)EB >= (int64_t(64) << 20)) ? 1 : 3;
  p->tile_P = best.P;
  p->tile_LA = best.LA;
  p->tile_LB = best.LB;
  p->tile_ntiles = ntiles;
  for (int d = 0; d < f.rank; ++d) p->tile_ext[d] = best.ext[d];
  if (p->shape_only) {
    p->vecA = wants_shifted_runs(best, EA, p->tuning) ? 16 / EA : best.vecA;
    p->shape_shifted = wants_shifted_runs(best, EA, p->tuning);
    p->shape_bulk = bulk_possible(best, EA, p->tuning, p->shape_shifted);
    p->vecB = best.vecB;
    p->est_cost = best.cost;
    // the staged kernel's ring depth and CTAs per SM, from the staged layout's usual size (the bank
    // padding adds about 6% to a tile; the exact size needs the full descriptor)
    int64_t nfull = 1;
    for (int d = 0; d < f.rank; ++d) {
      if (best.ext[d] == 0)
        nfull *= f.n[d];
      else if (best.ext[d] < f.n[d])
        nfull *= f.n[d] / best.ext[d];
    }
    const int64_t P = best.P, stage_elems = P + P / 16;
    const int EBb = dtype_bytes(p->tb);
    auto smem_for = [&](int S) {
      return (int64_t)ttcb::async_smem_bytes(S, (int)stage_elems, (int)P, (int)(P / best.LA), (int)(P / best.LB), EA,
                                             EBb, beta);
    };
    const StageChoice sc = choose_stages(P, EA, EBb, beta, p->vecA, best.vecB, nfull, smem_for, p->tuning.stages);
    p->shape_stages = sc.S;
    p->ctas_per_sm = p->tuning.ctas_per_sm > 0 ? p->tuning.ctas_per_sm : sc.c;
    return TTCB_OK;
  }
  build_tile_desc(p, best, EA);
  {
    // shifted A runs exist only for the staged kernel: when it cannot run this tile (or the schedule
    // names another tile kernel), the plan is made with the plain layout instead
    const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
    const int tv = p->tuning.tile_variant;
    if (td->shiftA && (!td->async_ok || (tv != 0 && tv != 3))) {
      p->tuning.shifted_runs = -1;
      build_tile_desc(p, best, EA);
    }
  }
  return TTCB_OK;
}

// ------------------------------------------------------------------------------------------------
// The ragged tiles of a tile plan cover the last block [start, n) of each ragged fused dimension:
// box 0 is that block of the first ragged dimension with every other dimension whole; box 1 is the
// last block of the second one with the first dimension below its start. Each box keeps the fused
// strides, written as TTC leading dimensions: consecutive fused strides divide each other (they are
// products of the caller's leading dimensions), and a unit dimension in front carries a first
// stride other than 1.
int plan_edge_boxes(const ttcb_plan* p, EdgeBox out[2]) {
  const FusedProblem& f = p->f;
  int n = 0;
  while (n < 2 && p->rag_dim[n] >= 0) ++n;
  if (n == 0) return 0;
  const int r = f.rank;
  const int s = (f.sA[0] != 1 || f.sB[f.perm[0]] != 1) ? 1 : 0;
  if (r + s > TTCB_MAXR) return -1;
  for (int k = 0; k < n; ++k) {
    int64_t lo[TTCB_MAXR], ext[TTCB_MAXR];
    for (int i = 0; i < r; ++i) {
      lo[i] = 0;
      ext[i] = f.n[i];
    }
    const int d = p->rag_dim[k];
    lo[d] = p->rag_start[k];
    ext[d] = f.n[d] - p->rag_start[k];
    if (k == 1) ext[p->rag_dim[0]] = p->rag_start[0];
    EdgeBox& b = out[k];
    b.offA = b.offB = 0;
    for (int i = 0; i < r; ++i) {
      b.offA += lo[i] * f.sA[i];
      b.offB += lo[i] * f.sB[i];
    }
    b.rank = r + s;
    if (s) {
      b.perm[0] = 0;
      b.size[0] = 1;
      b.lda[0] = f.sA[0];
      b.ldb[0] = f.sB[f.perm[0]];
    }
    for (int i = 0; i < r; ++i) {
      b.size[i + s] = ext[i];
      b.lda[i + s] = i + 1 < r ? f.sA[i + 1] / f.sA[i] : ext[i];
    }
    for (int j = 0; j < r; ++j) {
      b.perm[j + s] = f.perm[j] + s;
      b.ldb[j + s] = j + 1 < r ? f.sB[f.perm[j + 1]] / f.sB[f.perm[j]] : ext[f.perm[j]];
    }
  }
  return n;
}

std::string plan_describe_json(const ttcb_plan* p) {
  static const char* names[] = {"s", "d", "c", "z"};
  std::ostringstream o;
  o << "{\"rank\":" << p->rank << ",\"dtypeA\":\"" << names[p->ta] << "\",\"dtypeB\":\"" << names[p->tb]
    << "\",\"beta\":" << (p->beta_nonzero ? 1 : 0) << ",\"elements\":" << p->N;
  o << ",\"fused\":{\"rank\":" << p->f.rank << ",\"perm\":[";
  for (int i = 0; i < p->f.rank; ++i) o << (i ? "," : "") << p->f.perm[i];
  o << "],\"size\":[";
  for (int i = 0; i < p->f.rank; ++i) o << (i ? "," : "") << p->f.n[i];
  o << "],\"strideA\":[";
  for (int i = 0; i < p->f.rank; ++i) o << (i ? "," : "") << p->f.sA[i];
  o << "],\"strideB\":[";
  for (int i = 0; i < p->f.rank; ++i) o << (i ? "," : "") << p->f.sB[i];
  o << "]}";
  o << ",\"kernel\":\"" << (p->kernel == TTCB_KERNEL_TILE ? "tile" : p->kernel == TTCB_KERNEL_ROW ? "row" : "none")
    << "\",\"vecA\":" << p->vecA << ",\"vecB\":" << p->vecB << ",\"blocks\":" << p->blocks
    << ",\"streaming\":" << (p->streaming ? 1 : 0) << ",\"loop_order\":" << p->loop_order;
  o << ",\"raster\":[";
  for (int k = 0; k < p->nraster; ++k) o << (k ? "," : "") << p->raster[k];
  o << "]"
    << ",\"tile_variant\":" << p->tuning.tile_variant
    << ",\"smem\":" << p->smem_bytes << ",\"est_cost\":" << p->est_cost;
  if (p->kernel == TTCB_KERNEL_TILE && !p->host_desc.empty()) {
    const TileDesc* t = reinterpret_cast<const TileDesc*>(p->host_desc.data());
    o << ",\"tile\":{\"P\":" << t->P << ",\"LA\":" << t->LA << ",\"LB\":" << t->LB << ",\"ntiles\":" << t->ntiles
      << ",\"ngrid\":" << t->ngrid << ",\"nblocked\":" << t->nblocked << ",\"pad\":" << t->pad
      << ",\"pshift\":" << t->pshift << ",\"fast\":" << t->fast << ",\"async\":" << t->async_ok
      << ",\"padA\":" << t->padA << ",\"sigmaA\":" << t->sigmaA << ",\"stages\":" << t->nstages
      << ",\"reg\":" << t->reg_ok << ",\"smem_async\":" << p->smem_async
      << ",\"blocks_async\":" << p->blocks_async << ",\"ctas_per_sm\":" << p->ctas_per_sm
      << ",\"shifted_runs\":" << t->shiftA << ",\"bulk\":" << t->bulkA << ",\"lane_map\":" << (t->map_log2s >= 0 ? (1 << t->map_log2s) : 0) << ",\"claims\":" << (p->claim_words ? 1 : 0) << ",\"claim_group\":" << p->claim_group
      << ",\"ragged_tiles\":" << (t->nrag0 + t->nrag1) << ",\"ext\":[";
    for (int d = 0; d < p->f.rank; ++d) o << (d ? "," : "") << p->tile_ext[d];
    o << "]}";
  } else if (p->kernel == TTCB_KERNEL_TILE && p->shape_only) {
    const bool fits = p->tile_P / p->vecA <= 1024 && p->tile_P / p->vecB <= 1024;
    o << ",\"tile\":{\"P\":" << p->tile_P << ",\"LA\":" << p->tile_LA << ",\"LB\":" << p->tile_LB
      << ",\"ntiles\":" << p->tile_ntiles << ",\"fast\":" << (fits ? 1 : 0) << ",\"stages\":" << p->shape_stages
      << ",\"ctas_per_sm\":" << p->ctas_per_sm << ",\"shifted_runs\":" << (p->shape_shifted ? 1 : 0)
      << ",\"bulk\":" << (p->shape_bulk ? 1 : 0)
      << ",\"shape_only\":1,\"ext\":[";
    for (int d = 0; d < p->f.rank; ++d) o << (d ? "," : "") << p->tile_ext[d];
    o << "]}";
  } else if (p->kernel == TTCB_KERNEL_ROW && !p->host_desc.empty()) {
    const RowDesc* rd = reinterpret_cast<const RowDesc*>(p->host_desc.data());
    o << ",\"row\":{\"w\":" << rd->w << ",\"chunk\":" << rd->chunk << ",\"units\":" << rd->nunits << "}";
  }
  if (p->nedge > 0) {
    o << ",\"edges\":[";
    for (int k = 0; k < p->nedge; ++k)
      o << (k ? "," : "") << "{\"offA\":" << p->edge[k]->base_offA << ",\"offB\":" << p->edge[k]->base_offB
        << ",\"plan\":" << plan_describe_json(p->edge[k]) << "}";
    o << "]";
  }
  o << "}";
  return o.str();
}
