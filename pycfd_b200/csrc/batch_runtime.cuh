// Host runtime of the batched step (pycfd_batch_*).  Compiled inside
// solver.cu's translation unit: a batch keeps one single-problem solver per
// problem for its geometry, boundary table, scalar block and vectors, and uses
// the solver's upload helpers for the shared multigrid hierarchies.
#pragma once
#include <climits>

#include "batch.cuh"

namespace {

struct BMapHost {
  int2* e = nullptr;   // device
  int n = 0;
};

}  // namespace

struct pycfd_batch {
  int n = 0;
  int precision = PCFD_FP64;
  double tol = 1e-10, inner_tol = 1e-4;
  int maxiter = 1000, sweeps = 1, tile_i = 32;
  int coarse = 0;                          // levels >= coarse: one block per problem (0: per level)
  int fused = 0;                           // down sweep by fused restrictions (every structure has them)
  int fused_from = 1;                      // first level restricted by the fused product (1 or 2)
  int ell_group = kBGroup;                 // problems per block of the coarse-level launches (1 or kBGroup)
  int stencil_req = 0;                     // level-0 transfers as stencils, as asked
  int stencil = 0;                         // ... and in force (fused down sweep from the fine level)
  int scalar_strips = 0;                   // FP32 solver kernels on scalar strips even where rows allow vectors
  int* order = nullptr;                    // problems by size, largest first (coarse kernel)
  std::vector<pycfd_solver*> solvers;
  pycfd_solver* mem = nullptr;             // owner of the batch's own device allocations
  void* probs = nullptr;                   // BProb<T>[n] (device)
  void* hiers = nullptr;                   // BHier<T>[nh] (device)
  std::vector<int> nlev;
  int depth = 0;                           // most levels of any problem
  BMapHost fine;                           // every chunk of tiles of every problem
  BMapHost strip;                          // every chunk of warp strips of every problem (solver kernels)
  BMapHost vstrip;                         // the CG and level-0 sweep kernels: vector chunks where in force
  BMapHost halo;                           // every staged tile of every problem (stencil transfers)
  BMapHost pstrip;                         // every chunk of predictor strips of every problem
  // row-block maps per depth d (problems whose level d runs per level):
  // grouped maps per depth d, entries (structure, row block x 1024 + group of ell_group problems):
  std::vector<BMapHost> mapA;              // smoothing/residual with A_d (d >= 1)
  std::vector<BMapHost> mapR;              // restriction into d
  std::vector<BMapHost> mapP;              // prolongation into d with P_{d+1}
  std::vector<BMapHost> mapC;              // (problem, -1): coarsest level d of an untailed structure
  BMapHost mapT;                           // dense tails: (structure, row block x 64 + problem group)
  int* sprobs = nullptr;                   // problems grouped by structure
  size_t smem_dense = 0;
  BShared sh{};
  int* h_any = nullptr;                    // pinned mirror of sh.any
  long long* h_passes = nullptr;           // pinned mirror of sh.passes
  int* d_iout = nullptr;
  double* d_dout = nullptr;
  // launches recorded per part of the step (launch accounting of replays)
  long long fixed_launches = 0, cg_body_launches = 0, ir_body_launches = 0;
  bool capturing = false;
  cudaStream_t aux = nullptr, aux2 = nullptr, rec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

constexpr int kIrMaxPassesB = 40;
constexpr int kInnerMaxIterB = 200;
constexpr int kBChunkCells = 4096;   // fine cells per block of a fine launch

int upload_map(pycfd_batch* B, BMapHost* m, const std::vector<int2>& h) {
  m->n = (int)h.size();
  if (h.empty()) return 0;
  return upload(B->mem, &m->e, h.data(), h.size());
}

// Upload one structure's hierarchy (from the descriptor of its first problem)
// in storage type T.
template <class T>
int upload_hier(pycfd_batch* B, const pycfd_solver_desc* d, BHier<T>* H, std::vector<Level>* keep) {
  const int Lv = d->n_levels;
  keep->resize(Lv);
  H->nlev = Lv;
  H->w0 = d->levels[0].weight;
  H->agg2 = Lv >= 2 && d->levels[1].shape_x == (d->nx + 1) / 2 && d->levels[1].shape_y == (d->ny + 1) / 2 &&
            d->levels[1].n == d->levels[1].shape_x * d->levels[1].shape_y;
  for (int l = 1; l < Lv; ++l) {
    const pycfd_mg_level& in = d->levels[l];
    const pycfd_mg_level& up = d->levels[l - 1];
    Level& L = (*keep)[l];
    L.n = in.n;
    const bool coarsest = l == Lv - 1;
    DevEll<T> A, P, R;
    T* wd = nullptr;
    if (!coarsest) {
      if (!in.a_indptr || !in.weighted_dinv) return fail(PCFD_E_ARG, "level %d lacks A", l);
      TRY(make_ell(B->mem, &A, in.n, in.a_indptr, in.a_indices, in.a_data));
      std::vector<T> w(in.weighted_dinv, in.weighted_dinv + in.n);
      TRY(upload(B->mem, &wd, w.data(), w.size()));
    }
    if (!in.p_indptr) return fail(PCFD_E_ARG, "level %d lacks P", l);
    TRY(make_ell(B->mem, &P, up.n, in.p_indptr, in.p_indices, in.p_data));
    std::vector<int64_t> tp;
    std::vector<int32_t> ti;
    std::vector<double> td;
    csr_transpose(up.n, in.n, in.p_indptr, in.p_indices, in.p_data, tp, ti, td);
    TRY(make_ell(B->mem, &R, in.n, tp.data(), ti.data(), td.data()));
    BLevel<T>& bl = H->lv[l];
    if (in.m_indptr) {
      DevEll<T> M;
      TRY(make_ell(B->mem, &M, in.n, in.m_indptr, in.m_indices, in.m_data));
      bl.M = M.view();
      bl.lm = M.lanes;
    }
    bl.A = A.view();
    bl.la = A.lanes;
    bl.P = P.view();
    bl.lp = P.lanes;
    bl.R = R.view();
    bl.lr = R.lanes;
    bl.wd = wd;
    bl.n = in.n;
  }
  if (B->coarse == 0 && d->tail_level > 0 && d->tail_level < Lv - 1 && d->tail_operator) {
    const int nt = d->levels[d->tail_level].n;
    std::vector<T> m((size_t)nt * nt);
    for (size_t e = 0; e < m.size(); ++e) m[e] = (T)d->tail_operator[e];
    T* md = nullptr;
    TRY(upload(B->mem, &md, m.data(), m.size()));
    H->tail = md;
    H->tail_level = d->tail_level;
    H->tail_n = nt;
    H->fused = 1;
    for (int l = 1; l <= d->tail_level; ++l)
      if (!d->levels[l].m_indptr) H->fused = 0;
  }
  const int nc = d->levels[Lv - 1].n;
  std::vector<T> c((size_t)nc * nc);
  for (size_t e = 0; e < c.size(); ++e) c[e] = (T)d->coarsest_inverse[e];
  T* cd = nullptr;
  TRY(upload(B->mem, &cd, c.data(), c.size()));
  H->C = cd;
  H->nc = nc;
  B->smem_dense = std::max(B->smem_dense, (size_t)nc * sizeof(double));
  return 0;
}

template <class T>
int batch_build(pycfd_batch* B, const pycfd_solver_desc* descs, const int* structure,
                const pycfd_dt_control* ctl, const int* max_steps, double* const* u, double* const* v,
                double* const* p) {
  const int n = B->n;
  // hierarchies: one per structure (the problem that first names it)
  std::vector<int> hid(n, -1), leaders;
  for (int i = 0; i < n; ++i) {
    const int s = structure ? structure[i] : i;
    if (s < 0 || s > i) return fail(PCFD_E_ARG, "structure[%d] = %d must name this or an earlier problem", i, s);
    if (s == i) {
      hid[i] = (int)leaders.size();
      leaders.push_back(i);
    } else {
      if (structure[s] != s) return fail(PCFD_E_ARG, "structure[%d] must name a problem that leads its structure", i);
      if (descs[s].nx != descs[i].nx || descs[s].ny != descs[i].ny)
        return fail(PCFD_E_ARG, "problems %d and %d share a structure but not a grid", s, i);
      hid[i] = hid[s];
    }
  }
  std::vector<BHier<T>> hh(leaders.size());
  std::vector<std::vector<Level>> keep(leaders.size());
  for (size_t h = 0; h < leaders.size(); ++h) {
    const pycfd_solver_desc& d = descs[leaders[h]];
    if (d.n_levels < 2 || !d.levels || !d.coarsest_inverse)
      return fail(PCFD_E_ARG, "problem %d: the batched solve needs a multigrid hierarchy of at least 2 levels",
                  leaders[h]);
    if (d.n_levels > kBMaxLevels) return fail(PCFD_E_ARG, "at most %d multigrid levels", kBMaxLevels);
    if (d.levels[0].n != d.nx * d.ny) return fail(PCFD_E_ARG, "level 0 must have nx*ny unknowns");
    hh[h] = BHier<T>{};
    TRY(upload_hier<T>(B, &d, &hh[h], &keep[h]));
  }
  if (B->smem_dense > 48 * 1024)
    return fail(PCFD_E_UNSUPPORTED, "coarsest level too large for the one-block dense solve");

  // per-problem records
  std::vector<BProb<T>> pr(n);
  std::vector<int2> fine, strip, vstrip, pstrip, halo;
  B->nlev.assign(n, 0);
  B->depth = 0;
  int red_rows = 0;
  for (int i = 0; i < n; ++i) {
    pycfd_solver* s = B->solvers[i];
    BProb<T>& P = pr[i];
    P = BProb<T>{};
    P.g = s->g;
    P.bc = s->bc;
    const pycfd_dt_control& c = ctl[i];
    P.dtc = DtControl{c.adaptive, c.cfl, c.visc_limit, c.dt_cap, c.t_end, s->g.dx, s->g.dy, c.blend_mode, c.blend};
    P.hier = hid[i];
    P.nlev = descs[leaders[hid[i]]].n_levels;
    P.tail = hh[hid[i]].tail_level;
    B->nlev[i] = P.nlev;
    B->depth = std::max(B->depth, P.nlev);
    P.singular = s->singular;
    P.max_steps = max_steps ? max_steps[i] : INT_MAX;
    P.tile_i = B->tile_i;
    P.tiles_i = (s->g.nx + B->tile_i - 1) / B->tile_i;
    P.tiles_j = (s->g.ny + kBTileJ - 1) / kBTileJ;
    P.tiles = P.tiles_i * P.tiles_j;
    P.chunk_tiles = std::max(1, kBChunkCells / (B->tile_i * kBTileJ));
    P.chunks = (P.tiles + P.chunk_tiles - 1) / P.chunk_tiles;
    P.s_segs = (s->g.ny + kBSegCols - 1) / kBSegCols;
    P.s_items = ((s->g.nx + kBStripRows - 1) / kBStripRows) * P.s_segs;
    P.s_chunks = (P.s_items + kBStripItems - 1) / kBStripItems;
    P.v_chunks = (s->g.nx + kBVecRows - 1) / kBVecRows;
    {
      const int segs = (s->g.ny + 3 + kBPredCols - 1) / kBPredCols;
      const int items = segs * ((s->g.nx + 3 + kBStripRows - 1) / kBStripRows);
      P.p_chunks = (items + kBStripItems - 1) / kBStripItems;
    }
    {
      // staged tiles of the stencil transfers: as few row bands as the most rows
      // allow, of even height (aggregates pair rows)
      const int most = b_halo_tr_max<T>();
      const int bands = (s->g.nx + most - 1) / most;
      int tr = (s->g.nx + bands - 1) / bands;
      tr += tr & 1;
      P.h_tr = tr;
      P.h_tiles_j = (s->g.ny + kBHaloTC - 1) / kBHaloTC;
      P.h_tiles = ((s->g.nx + tr - 1) / tr) * P.h_tiles_j;
    }
    P.red_base = red_rows;
    red_rows += std::max(std::max(P.chunks, std::max(P.s_chunks, P.v_chunks)), P.h_tiles);
    P.flags = s->flags;
    P.solid = s->solid;
    P.bc_kind = s->bc_kind_dev;
    P.u = u[i];
    P.v = v[i];
    P.p = p[i];
    P.us1 = s->us1;
    P.vs1 = s->vs1;
    P.us2 = s->us2;
    P.vs2 = s->vs2;
    P.S = s->S;
    P.I = s->I;
    P.counter = s->counter;
    P.b = s->b;
    P.x = s->x;
    if (sizeof(T) == sizeof(double)) {
      P.xs = (T*)s->x;
      P.r = (T*)s->r;
      P.z = (T*)s->z;
      P.pa = (T*)s->pa;
      P.pb = (T*)s->pb;
      P.q = (T*)s->q;
    } else {
      P.xs = (T*)s->x32;
      P.r = (T*)s->r32;
      P.z = (T*)s->z32;
      P.pa = (T*)s->pa32;
      P.pb = (T*)s->pb32;
      P.q = (T*)s->q32;
    }
    const int nc0 = s->g.nx * s->g.ny;
    TRY(dalloc(B->mem, &P.lxa[0], nc0));
    TRY(dalloc(B->mem, &P.lxb[0], nc0));
    TRY(dalloc(B->mem, &P.lres[0], nc0));
    {
      // vector strips: FP32 vectors, rows a multiple of 4 long, every vector the
      // kernels read or write as float4 16-byte aligned (flags 4-byte aligned)
      auto a16 = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
      const bool al = a16(P.xs) && a16(P.r) && a16(P.z) && a16(P.pa) && a16(P.pb) && a16(P.q) &&
                      a16(P.lxa[0]) && a16(P.lxb[0]) && a16(P.lres[0]) && ((uintptr_t)P.flags & 3u) == 0;
      P.vec = (sizeof(T) == 4 && !B->scalar_strips && s->g.ny % 4 == 0 && al) ? 1 : 0;
    }
    const std::vector<Level>& K = keep[hid[i]];
    for (int l = 1; l < P.nlev; ++l) {
      TRY(dalloc(B->mem, &P.lb[l], K[l].n));
      TRY(dalloc(B->mem, &P.lxa[l], K[l].n));
      TRY(dalloc(B->mem, &P.lxb[l], K[l].n));
      TRY(dalloc(B->mem, &P.lres[l], K[l].n));
    }
    P.w0 = hh[hid[i]].w0;
    // diagonal per face-flag pattern: fine_diag's subtractions in its order (an
    // interior cell gets no Dirichlet terms), and w / diag as in fine_wdinv
    P.any_dir = s->g.dir_w || s->g.dir_e || s->g.dir_s || s->g.dir_n;
    for (int f = 0; f < 16; ++f) {
      double dg = 0.0;
      if (f & F_W) dg -= s->g.cx;
      if (f & F_E) dg -= s->g.cx;
      if (f & F_S) dg -= s->g.cy;
      if (f & F_N) dg -= s->g.cy;
      P.dtab[f] = dg;
      P.wtab[f] = dg != 0.0 ? P.w0 * (1.0 / dg) : 0.0;
    }
    P.C = hh[hid[i]].C;
    for (int l = 0; l < kBMaxLevels; ++l) P.lv[l] = hh[hid[i]].lv[l];
    for (int c = 0; c < P.chunks; ++c) fine.push_back(make_int2(i, c));
    for (int c = 0; c < P.s_chunks; ++c) strip.push_back(make_int2(i, c));
    for (int c = 0, nc = P.vec ? P.v_chunks : P.s_chunks; c < nc; ++c) vstrip.push_back(make_int2(i, c));
    for (int c = 0; c < P.h_tiles; ++c) halo.push_back(make_int2(i, c));
    for (int c = 0; c < P.p_chunks; ++c) pstrip.push_back(make_int2(i, c));
  }
  TRY(upload_map(B, &B->fine, fine));
  TRY(upload_map(B, &B->strip, strip));
  TRY(upload_map(B, &B->vstrip, vstrip));
  TRY(upload_map(B, &B->halo, halo));
  TRY(upload_map(B, &B->pstrip, pstrip));
  // problems grouped by structure (the dense tail's block groups)
  {
    std::vector<int> sp;
    for (size_t h = 0; h < leaders.size(); ++h) {
      hh[h].sp0 = (int)sp.size();
      for (int i = 0; i < n; ++i)
        if (hid[i] == (int)h) sp.push_back(i);
      hh[h].spn = (int)sp.size() - hh[h].sp0;
    }
    TRY(upload(B->mem, &B->sprobs, sp.data(), sp.size()));
    void* hd = nullptr;
    TRY(upload(B->mem, (uint8_t**)&hd, (const uint8_t*)hh.data(), hh.size() * sizeof(BHier<T>)));
    B->hiers = hd;
  }
  // row-block maps per depth: a block takes kBEllRounds x kBThreads / L rows
  // (L: lanes of its matrix).  With the coarse kernel, a problem's levels from
  // min(coarse, coarsest) on run there and take no per-level blocks.  A problem
  // whose structure has a dense tail at depth t takes the restriction into t
  // and no level below it; the tail blocks cover t.
  // fused down sweep: every structure closes its cycle with a tail and carries
  // the fused restrictions above it, one sweep per level
  B->fused = (B->coarse == 0 && B->sweeps == 1) ? 1 : 0;
  for (size_t h = 0; h < leaders.size(); ++h)
    if (!hh[h].fused || hh[h].tail_level == 0) B->fused = 0;
  // level-0 transfers as stencils: they stand for P_1 and M_1 of the 2 x 2
  // aggregation, so every structure must have that level 1
  B->stencil = (B->stencil_req && B->fused && B->fused_from == 1) ? 1 : 0;
  for (size_t h = 0; B->stencil && h < leaders.size(); ++h)
    if (!hh[h].agg2)
      return fail(PCFD_E_UNSUPPORTED, "stencil transfers: structure %d's level 1 is not the 2 x 2 aggregation",
                  (int)h);
  B->mapA.assign(B->depth, BMapHost{});
  B->mapR.assign(B->depth, BMapHost{});
  B->mapP.assign(B->depth, BMapHost{});
  B->mapC.assign(B->depth, BMapHost{});
  std::vector<int2> mt;
  for (int d = 0; d < B->depth; ++d) {
    std::vector<int2> ma, mr, mp, mc;
    for (size_t h = 0; h < leaders.size(); ++h) {
      const BHier<T>& H = hh[h];
      const int gs = B->ell_group;
      const int grps = (H.spn + gs - 1) / gs;
      if (grps > 1024) return fail(PCFD_E_UNSUPPORTED, "at most %d problems share a structure", 1024 * gs);
      if (H.tail_level == d && H.tail_n > 0) {
        const int rts = (H.tail_n + kTailBM - 1) / kTailBM;
        const int cts = (H.spn + kTailBN - 1) / kTailBN;
        for (int rt = 0; rt < rts; ++rt)
          for (int c = 0; c < cts; ++c) mt.push_back(make_int2((int)h, rt * 64 + c));
      }
      const int lead = leaders[h];
      const int c = B->nlev[lead] - 1;
      const int t = pr[lead].tail;
      if (B->coarse > 0) {
        if (d >= std::min(B->coarse, c)) continue;
      } else if (t > 0) {
        if (d > t) continue;
      } else {
        if (d > c) continue;
        if (d == c) {
          if (d >= 1)
            for (int i = 0; i < n; ++i)
              if (hid[i] == (int)h) mc.push_back(make_int2(i, -1));
          continue;
        }
      }
      const int nrow = d == 0 ? pr[lead].g.nx * pr[lead].g.ny : keep[h][d].n;
      auto add = [&](std::vector<int2>& m, int lanes) {
        const int rpb = kBThreads / lanes * (gs == 1 ? b_ell_rounds<1>() : b_ell_rounds<kBGroup>());
        for (int rb = 0; rb * rpb < nrow; ++rb)
          for (int g = 0; g < grps; ++g) m.push_back(make_int2((int)h, rb * 1024 + g));
      };
      const int lres = (B->fused && d >= B->fused_from) ? H.lv[d].lm : H.lv[d].lr;   // lanes of the restriction into d
      if (t > 0 && d == t) {   // restriction into the tail level only
        add(mr, lres);
        continue;
      }
      add(mp, H.lv[d + 1].lp);
      if (d >= 1) {
        add(ma, H.lv[d].la);
        add(mr, lres);
      }
    }
    TRY(upload_map(B, &B->mapA[d], ma));
    TRY(upload_map(B, &B->mapR[d], mr));
    TRY(upload_map(B, &B->mapP[d], mp));
    TRY(upload_map(B, &B->mapC[d], mc));
  }
  TRY(upload_map(B, &B->mapT, mt));
  {
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
      return (long)pr[a].g.nx * pr[a].g.ny > (long)pr[b].g.nx * pr[b].g.ny;
    });
    TRY(upload(B->mem, &B->order, ord.data(), ord.size()));
  }
  void* pd = nullptr;
  TRY(upload(B->mem, (uint8_t**)&pd, (const uint8_t*)pr.data(), pr.size() * sizeof(BProb<T>)));
  B->probs = pd;
  TRY(dalloc(B->mem, &B->sh.partials, (size_t)red_rows * 8));
  TRY(dalloc(B->mem, &B->sh.tickets, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.any, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.passes, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.iters, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.capped, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.cap_set, TK_COUNT));
  TRY(dalloc(B->mem, &B->sh.frozen, n));
  TRY(dalloc(B->mem, &B->sh.solving, n));
  TRY(dalloc(B->mem, &B->d_iout, (size_t)4 * n));
  TRY(dalloc(B->mem, &B->d_dout, (size_t)2 * n));
  return 0;
}

// ---- launches ----------------------------------------------------------------
// Every batched kernel starts with pdl_begin (waits for its predecessor's grid
// and memory), so with B->mem->pdl set a launch carries the programmatic-
// serialization attribute and its blocks are scheduled while the predecessor
// drains; with it clear (the default) the launches keep plain stream order.
#define BLAUNCH(kernel, grid, block, smem, stream, ...)                                    \
  do {                                                                                      \
    pdl_launch(B->mem, kernel, dim3(grid), dim3(block), (size_t)(smem), (stream), __VA_ARGS__); \
    CHECK_LAUNCH();                                                                         \
  } while (0)

const dim3 kBFineBlock(kBTileJ, kBThreadsI);

// Event pair around eager launches of one kernel kind (measurement support;
// ids: 1 k_b_cg_pq, 2 last fine V-cycle sweep, 3 first fine sweep, 4 coarse
// levels (ELL phases and the per-problem coarse block), 5 k_b_cg_xr, 6 predictor).
inline void b_prof(pycfd_batch* B, int id, cudaStream_t st) {
  if (id != 0 && !B->capturing) prof_mark(B->mem, id, st);
}

template <class T>
const BProb<T>* probs_of(pycfd_batch* B) { return (const BProb<T>*)B->probs; }
template <class T>
const BHier<T>* hiers_of(pycfd_batch* B) { return (const BHier<T>*)B->hiers; }

template <class T>
int b_boundary(pycfd_batch* B, int arr, std::initializer_list<int> ops, int p_ghosts, cudaStream_t st) {
  BcProgram prog{};
  int k = 0;
  for (int op : ops) prog.op[k++] = op;
  prog.op[k] = OP_END;
  BLAUNCH(k_b_boundary<T>, B->n, kBThreads, 0, st, probs_of<T>(B), arr, prog, p_ghosts, B->sh);
  return 0;
}

// One grouped ELL op at depth d; a restriction also closes the untailed
// structures whose coarsest level is d (restriction + dense solve per problem).
template <class T, int OP>
int b_ell(pycfd_batch* B, const BMapHost& m, int d, int src, int dst, cudaStream_t st) {
  const BMapHost* mc = (OP == EO_RESTRICT && d < (int)B->mapC.size()) ? &B->mapC[d] : nullptr;
  if (m.n == 0 && !(mc && mc->n)) return 0;
  b_prof(B, 4, st);
  if (m.n && B->ell_group == 1)
    BLAUNCH((k_b_ellg<T, OP, 1>), m.n, kBThreads, 0, st, probs_of<T>(B), hiers_of<T>(B), m.e, B->sprobs, d, src,
            dst, B->sh);
  else if (m.n)
    BLAUNCH((k_b_ellg<T, OP, kBGroup>), m.n, kBThreads, 0, st, probs_of<T>(B), hiers_of<T>(B), m.e, B->sprobs, d,
            src, dst, B->sh);
  if (mc && mc->n) BLAUNCH(k_b_coarsest<T>, mc->n, kBThreads, B->smem_dense, st, probs_of<T>(B), mc->e, d, B->sh);
  b_prof(B, 4, st);
  return 0;
}

template <class T, int MODE>
int b_fine(pycfd_batch* B, int src, int dst, cudaStream_t st) {
  const int id = MODE == FM_LAST ? 2 : MODE == FM_PRE ? 3 : 0;
  b_prof(B, id, st);
  BLAUNCH((k_b_fine<T, MODE>), B->vstrip.n, kBThreads, 0, st, probs_of<T>(B), hiers_of<T>(B), B->vstrip.e, src,
          dst, B->sh);
  b_prof(B, id, st);
  return 0;
}

// Level-0 transfers as stencils over every problem's staged tiles: the fused
// restriction into level 1 (up = false) or the prolongation from level 1 with
// the last fine sweep (up = true).
template <class T>
int b_stencil_transfer(pycfd_batch* B, bool up, cudaStream_t st) {
  const int id = up ? 2 : 3;
  b_prof(B, id, st);
  if (up) BLAUNCH(k_b_prolong_last<T>, B->halo.n, kBThreads, 0, st, probs_of<T>(B), B->halo.e, B->sh);
  else BLAUNCH(k_b_frestrict0<T>, B->halo.n, kBThreads, 0, st, probs_of<T>(B), B->halo.e, B->sh);
  b_prof(B, id, st);
  return 0;
}

// The dense tails of every tailed structure, one launch after the down sweep
// (each block reads its structure's tail depth).
template <class T>
int b_tails(pycfd_batch* B, cudaStream_t st) {
  if (B->mapT.n == 0) return 0;
  b_prof(B, 4, st);
  BLAUNCH(k_b_tail<T>, B->mapT.n, kTailThreads, 0, st, probs_of<T>(B), hiers_of<T>(B), B->mapT.e, B->sprobs,
          B->sh);
  b_prof(B, 4, st);
  return 0;
}

// One V-cycle from zero on every solving problem, levels in lockstep by depth:
// z <- M r, with mean(z) and r.z left in each problem's scalar block.  With
// B->coarse > 0 the levels from there down run in one block per problem.
template <class T>
int b_vcycle(pycfd_batch* B, cudaStream_t st) {
  const int sw = B->sweeps;
  const int D = B->coarse > 0 ? std::min(B->coarse, B->depth) : B->depth;   // depths run per level
  if (B->fused) {
    // ---- down: b_d = M_d b_{d-1} at every depth from fused_from above each problem's
    // tail (below it the fine sweep and R), then the tails
    const bool fine_kept = B->fused_from == 2;
    if (fine_kept) TRY((b_fine<T, FM_PRE>(B, 0, 0, st)));
    for (int d = 1; d < D; ++d) {
      if (d < B->fused_from) TRY((b_ell<T, EO_RESTRICT>(B, B->mapR[d], d, 0, 0, st)));
      else if (d == 1 && B->stencil) TRY(b_stencil_transfer<T>(B, false, st));
      else TRY((b_ell<T, EO_FRESTRICT>(B, B->mapR[d], d, 0, 0, st)));
    }
    TRY(b_tails<T>(B, st));
    // ---- up: x_d = W b_d + P x_{d+1} into xa, one sweep into xb
    for (int d = D - 2; d >= 1; --d) {
      if (B->mapA[d].n == 0) continue;
      TRY((b_ell<T, EO_PROLONGW>(B, B->mapP[d], d, 1, 0, st)));
      TRY((b_ell<T, EO_SMOOTH>(B, B->mapA[d], d, 0, 1, st)));
    }
    if (B->stencil) return b_stencil_transfer<T>(B, true, st);   // prolongation and last sweep in one pass
    if (fine_kept) TRY((b_ell<T, EO_PROLONG>(B, B->mapP[0], 0, 1, 0, st)));   // x_0 stored by FM_PRE
    else TRY((b_ell<T, EO_PROLONGW>(B, B->mapP[0], 0, 1, 0, st)));
    TRY((b_fine<T, FM_LAST>(B, 0, 2, st)));
    return 0;
  }
  // ---- down ----
  int cur0 = 0;
  if (sw == 1) {
    TRY((b_fine<T, FM_PRE>(B, 0, 0, st)));
  } else {
    TRY((b_fine<T, FM_WDB>(B, 0, 0, st)));
    int a = 0, o = 1;
    for (int k = 1; k < sw; ++k) {
      TRY((b_fine<T, FM_SMOOTH>(B, a, o, st)));
      std::swap(a, o);
    }
    TRY((b_fine<T, FM_RESID>(B, a, a, st)));
    cur0 = a;
  }
  std::vector<int> cur(B->depth + 1, 0), fin(B->depth + 1, 0);
  for (int d = 1; d < D; ++d) {
    TRY((b_ell<T, EO_RESTRICT>(B, B->mapR[d], d, 0, 0, st)));
    if (B->mapA[d].n == 0) continue;
    TRY((b_ell<T, EO_PRE>(B, B->mapA[d], d, 0, 0, st)));
    int a = 0, o = 1;
    if (sw > 1) {
      for (int k = 1; k < sw; ++k) {
        TRY((b_ell<T, EO_SMOOTH>(B, B->mapA[d], d, a, o, st)));
        std::swap(a, o);
      }
      TRY((b_ell<T, EO_RESID>(B, B->mapA[d], d, a, a, st)));
    }
    cur[d] = a;
  }
  TRY(b_tails<T>(B, st));
  if (B->coarse > 0) {
    b_prof(B, 4, st);
    BLAUNCH(k_b_coarse<T>, B->n, kBCoarseThreads, B->smem_dense, st, probs_of<T>(B), B->order, B->coarse, sw,
            B->sh);
    b_prof(B, 4, st);
    fin[D] = b_coarse_final(sw);
  }
  // ---- up ----
  for (int d = D - (B->coarse > 0 ? 1 : 2); d >= 1; --d) {
    if (B->mapA[d].n == 0) continue;
    TRY((b_ell<T, EO_PROLONG>(B, B->mapP[d], d, fin[d + 1], cur[d], st)));
    int xf = cur[d], o = 1 - cur[d];
    for (int k = 1; k <= sw; ++k) {
      TRY((b_ell<T, EO_SMOOTH>(B, B->mapA[d], d, xf, o, st)));
      std::swap(xf, o);
    }
    fin[d] = xf;
  }
  TRY((b_ell<T, EO_PROLONG>(B, B->mapP[0], 0, fin[1], cur0, st)));
  int xf = cur0, o = 1 - cur0;
  for (int k = 1; k <= sw; ++k) {
    if (k == sw) {
      TRY((b_fine<T, FM_LAST>(B, xf, 2, st)));
    } else {
      TRY((b_fine<T, FM_SMOOTH>(B, xf, o, st)));
      std::swap(xf, o);
    }
  }
  return 0;
}

// ---- device-side loops ---------------------------------------------------------
int b_read_any(pycfd_batch* B, int site, cudaStream_t st, int* any) {
  CU(cudaMemcpyAsync(B->h_any, B->sh.any, sizeof(int) * TK_COUNT, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  *any = B->h_any[site];
  return 0;
}

int b_loop_handle(cudaStream_t st, cudaGraph_t* owner, LoopCtl* ctl) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  CU(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
  cudaGraphConditionalHandle h;
  CU(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  *ctl = LoopCtl{h, 1};
  if (owner) *owner = g;
  return 0;
}

// Append a WHILE node after the work captured on `st`; its body is then
// recorded on `body_st` until b_loop_close.
int b_loop_open(cudaStream_t st, cudaStream_t body_st, const LoopCtl& ctl) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CU(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = ctl.handle;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CU(cudaGraphAddNode(&node, g, deps, nd, &np));
  CU(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  CU(cudaStreamBeginCaptureToGraph(body_st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                   cudaStreamCaptureModeRelaxed));
  return 0;
}

int b_loop_close(cudaStream_t body_st) {
  cudaGraph_t out = nullptr;
  CU(cudaStreamEndCapture(body_st, &out));
  return 0;
}

// ---- solves ------------------------------------------------------------------------
// FP64 MG-PCG on every problem: x from the warm start, normalised result in x.
int b_solve_fp64(pycfd_batch* B, cudaStream_t st) {
  using T = double;
  const BProb<T>* P = probs_of<T>(B);
  LoopCtl ctl{0, 0};
  if (B->capturing) TRY(b_loop_handle(st, nullptr, &ctl));
  BLAUNCH(k_b_rhs_init<T>, B->strip.n, kBThreads, 0, st, P, B->n, B->strip.e, B->tol, B->maxiter, B->sh, ctl);
  auto pass = [&](cudaStream_t s2) -> int {
    TRY(b_vcycle<T>(B, s2));
    b_prof(B, 1, s2);
    BLAUNCH(k_b_cg_pq<T>, B->vstrip.n, kBThreads, 0, s2, P, B->vstrip.e, B->sh);
    b_prof(B, 1, s2);
    b_prof(B, 5, s2);
    BLAUNCH(k_b_cg_xr<T>, B->vstrip.n, kBThreads, 0, s2, P, B->n, B->vstrip.e, B->maxiter, B->sh, ctl);
    b_prof(B, 5, s2);
    return 0;
  };
  if (B->capturing) {
    TRY(b_loop_open(st, B->aux, ctl));
    const long long l0 = g_launches.load();
    TRY(pass(B->aux));
    B->cg_body_launches = g_launches.load() - l0;
    TRY(b_loop_close(B->aux));
  } else {
    for (int guard = 0; guard <= B->maxiter; ++guard) {
      int any = 0;
      TRY(b_read_any(B, TK_CG, st, &any));
      if (!any) break;
      TRY(pass(st));
    }
  }
  BLAUNCH(k_b_finish_stats<T>, B->strip.n, kBThreads, 0, st, P, B->strip.e, B->tol, B->sh);
  BLAUNCH(k_b_finish_apply<T>, B->strip.n, kBThreads, 0, st, P, B->strip.e, B->sh);
  return 0;
}

// Mixed form: FP64 iterative refinement around FP32 MG-PCG inner solves.
int b_solve_mixed(pycfd_batch* B, cudaStream_t st) {
  using T = float;
  const BProb<T>* P = probs_of<T>(B);
  LoopCtl outer{0, 0}, inner{0, 0};
  if (B->capturing) TRY(b_loop_handle(st, nullptr, &outer));
  BLAUNCH(k_b_ir_residual<T>, B->strip.n, kBThreads, 0, st, P, B->n, B->strip.e, B->tol, B->inner_tol,
          kIrMaxPassesB, 1, B->sh, outer);
  auto inner_pass = [&](cudaStream_t s2) -> int {
    TRY(b_vcycle<T>(B, s2));
    b_prof(B, 1, s2);
    BLAUNCH(k_b_cg_pq<T>, B->vstrip.n, kBThreads, 0, s2, P, B->vstrip.e, B->sh);
    b_prof(B, 1, s2);
    b_prof(B, 5, s2);
    BLAUNCH(k_b_cg_xr<T>, B->vstrip.n, kBThreads, 0, s2, P, B->n, B->vstrip.e, kInnerMaxIterB, B->sh, inner);
    b_prof(B, 5, s2);
    return 0;
  };
  auto refine = [&](cudaStream_t s2) -> int {
    BLAUNCH(k_b_ir_update<T>, B->strip.n, kBThreads, 0, s2, P, B->strip.e, B->sh);
    BLAUNCH(k_b_ir_residual<T>, B->strip.n, kBThreads, 0, s2, P, B->n, B->strip.e, B->tol, B->inner_tol,
            kIrMaxPassesB, 0, B->sh, outer);
    return 0;
  };
  if (B->capturing) {
    TRY(b_loop_open(st, B->aux, outer));
    const long long l0 = g_launches.load();
    cudaGraph_t body = nullptr;
    TRY(b_loop_handle(B->aux, &body, &inner));
    BLAUNCH(k_b_ir_arm<T>, 1, kBThreads, 0, B->aux, P, B->n, B->sh, inner);
    TRY(b_loop_open(B->aux, B->aux2, inner));
    const long long l1 = g_launches.load();
    TRY(inner_pass(B->aux2));
    B->cg_body_launches = g_launches.load() - l1;
    TRY(b_loop_close(B->aux2));
    TRY(refine(B->aux));
    B->ir_body_launches = g_launches.load() - l0 - B->cg_body_launches;
    TRY(b_loop_close(B->aux));
  } else {
    for (int g1 = 0; g1 <= kIrMaxPassesB + 1; ++g1) {
      int any = 0;
      TRY(b_read_any(B, TK_IR, st, &any));
      if (!any) break;
      BLAUNCH(k_b_ir_arm<T>, 1, kBThreads, 0, st, P, B->n, B->sh, inner);
      for (int g2 = 0; g2 <= kInnerMaxIterB; ++g2) {
        int a2 = 0;
        TRY(b_read_any(B, g2 == 0 ? TK_ARM : TK_CG, st, &a2));
        if (!a2) break;
        TRY(inner_pass(st));
      }
      TRY(refine(st));
    }
  }
  BLAUNCH(k_b_finish_stats<T>, B->strip.n, kBThreads, 0, st, P, B->strip.e, B->tol, B->sh);
  BLAUNCH(k_b_finish_apply<T>, B->strip.n, kBThreads, 0, st, P, B->strip.e, B->sh);
  return 0;
}

// Projection of stage array `arr` of every problem (pycfd/core/solver.py:643-683).
template <class T>
int b_project(pycfd_batch* B, int arr, cudaStream_t st) {
  const BProb<T>* P = probs_of<T>(B);
  BLAUNCH(k_b_div_rhs<T>, B->strip.n, kBThreads, 0, st, P, B->strip.e, arr, B->sh);
  if (B->precision == PCFD_MIXED) TRY(b_solve_mixed(B, st));
  else TRY(b_solve_fp64(B, st));
  BLAUNCH(k_b_correct<T>, B->fine.n, kBFineBlock, 0, st, P, B->fine.e, arr, B->sh);
  return 0;
}

// One projected Euler substep of every problem: stage input ca*a + cb*b into dst.
template <class T>
int b_substep(pycfd_batch* B, int a, int b, double ca, double cb, int dst, cudaStream_t st) {
  b_prof(B, 6, st);
  BLAUNCH(k_b_predictor<T>, B->pstrip.n, kBThreads, 0, st, probs_of<T>(B), B->pstrip.e, a, b, ca, cb, dst, B->sh);
  b_prof(B, 6, st);
  TRY(b_boundary<T>(B, dst, {OP_VEL_PRED, OP_MASS, OP_MASK_RESET, OP_WRAP_FACES}, 0, st));
  TRY(b_project<T>(B, dst, st));
  TRY(b_boundary<T>(B, dst, {OP_MASK_ACC, OP_WRAP_FACES, OP_VEL_CORR}, 1, st));
  return 0;
}

// One adaptive SSP-RK3 step of every unfrozen problem, in place
// (pycfd/core/solver.py:686-731, pycfd/core/timestepper.py:94-142).
template <class T>
int b_step(pycfd_batch* B, cudaStream_t st) {
  const BProb<T>* P = probs_of<T>(B);
  BLAUNCH(k_b_stats<T>, B->fine.n, kBFineBlock, 0, st, P, B->fine.e, B->sh);
  BLAUNCH(k_b_dt<T>, (B->n + 127) / 128, 128, 0, st, P, B->n, B->sh);
  TRY(b_substep<T>(B, 0, -1, 1.0, 0.0, 1, st));
  TRY(b_substep<T>(B, 1, -1, 1.0, 0.0, 2, st));
  TRY(b_substep<T>(B, 0, 2, 0.75, 0.25, 1, st));
  BLAUNCH(k_b_combine<T>, B->fine.n, kBFineBlock, 0, st, P, B->fine.e, 1, 1.0 / 3.0, 2.0 / 3.0, B->sh);
  TRY(b_boundary<T>(B, 0, {OP_VEL_CORR, OP_WRAP_FACES}, 0, st));
  return 0;
}

template <class T>
int b_initialize(pycfd_batch* B, cudaStream_t st) {
  BLAUNCH(k_b_set_dt<T>, (B->n + 127) / 128, 128, 0, st, probs_of<T>(B), B->n, 1.0);
  TRY(b_boundary<T>(B, 0, {OP_VEL_PRED, OP_MASS, OP_MASK_NONE, OP_WRAP_FACES}, 0, st));
  TRY(b_project<T>(B, 0, st));
  TRY(b_boundary<T>(B, 0, {OP_MASK_NONE, OP_WRAP_FACES, OP_VEL_CORR}, 1, st));
  return 0;
}

int b_dispatch_step(pycfd_batch* B, cudaStream_t st) {
  return B->precision == PCFD_MIXED ? b_step<float>(B, st) : b_step<double>(B, st);
}

}  // namespace

// ============================================================================
// C ABI (batched stepping)
// ============================================================================
extern "C" {

int pycfd_batch_destroy(pycfd_batch* B) {
  if (!B) return 0;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->aux) cudaStreamDestroy(B->aux);
  if (B->aux2) cudaStreamDestroy(B->aux2);
  if (B->rec) cudaStreamDestroy(B->rec);
  for (pycfd_solver* s : B->solvers) pycfd_solver_destroy(s);
  if (B->mem) pycfd_solver_destroy(B->mem);
  if (B->h_any) cudaFreeHost(B->h_any);
  if (B->h_passes) cudaFreeHost(B->h_passes);
  delete B;
  return 0;
}

int pycfd_batch_create(const pycfd_solver_desc* descs, const int* structure, const pycfd_dt_control* dt_ctl,
                       const int* max_steps, double* const* u, double* const* v, double* const* p, int n,
                       const pycfd_batch_opts* opts, pycfd_batch** out) {
  if (!descs || !dt_ctl || !u || !v || !p || !opts || !out || n < 1) return fail(PCFD_E_ARG, "bad arguments");
  if (opts->precision != PCFD_FP64 && opts->precision != PCFD_MIXED)
    return fail(PCFD_E_ARG, "precision must be PCFD_FP64 or PCFD_MIXED");
  if (opts->tile_rows != 8 && opts->tile_rows != 16 && opts->tile_rows != 32 && opts->tile_rows != 64)
    return fail(PCFD_E_ARG, "tile_rows must be 8, 16, 32 or 64");
  if (opts->mg_sweeps < 1 || opts->mg_sweeps > 4) return fail(PCFD_E_ARG, "mg_sweeps must be 1..4");
  if (opts->fused_from < 0 || opts->fused_from > 2) return fail(PCFD_E_ARG, "fused_from must be 0, 1 or 2");
  if (opts->ell_group != 0 && opts->ell_group != 1 && opts->ell_group != kBGroup)
    return fail(PCFD_E_ARG, "ell_group must be 0, 1 or %d", kBGroup);
  if (opts->coarse_level < 0 || opts->coarse_level >= kBMaxLevels)
    return fail(PCFD_E_ARG, "coarse_level must be 0..%d", kBMaxLevels - 1);
  if (!(opts->tol > 0) || opts->maxiter < 1) return fail(PCFD_E_ARG, "bad tolerance or iteration limit");
  for (int i = 0; i < n; ++i) {
    if (!u[i] || !v[i] || !p[i]) return fail(PCFD_E_ARG, "problem %d: null state pointer", i);
    if (descs[i].time_scheme != PCFD_RK3) return fail(PCFD_E_UNSUPPORTED, "the batched step is SSP-RK3");
  }
  pycfd_batch* B = new pycfd_batch();
  auto bail = [&](int rc) { pycfd_batch_destroy(B); return rc; };
  B->n = n;
  B->precision = opts->precision;
  B->tol = opts->tol;
  B->maxiter = opts->maxiter;
  B->inner_tol = opts->inner_tol > 0 ? opts->inner_tol : 1e-4;
  B->sweeps = opts->mg_sweeps;
  B->tile_i = opts->tile_rows;
  B->coarse = opts->coarse_level;
  B->fused_from = opts->fused_from == 2 ? 2 : 1;
  B->ell_group = opts->ell_group == 1 ? 1 : kBGroup;
  B->stencil_req = opts->stencil_transfer ? 1 : 0;
  B->scalar_strips = opts->scalar_strips ? 1 : 0;
  B->mem = new pycfd_solver();
  B->mem->pdl = opts->programmatic_launch ? 1 : 0;
  B->solvers.assign(n, nullptr);
  for (int i = 0; i < n; ++i) {
    // the single-problem record: geometry, masks, boundary table, scalars, vectors
    pycfd_solver_desc d = descs[i];
    d.solver_kind = PCFD_SOLVER_CG;
    d.n_levels = 0;
    d.levels = nullptr;
    d.coarsest_inverse = nullptr;
    d.coarse_cluster_rows = 0;
    d.persistent_solve = 0;
    d.tail_level = 0;
    d.tail_operator = nullptr;
    d.precision = opts->precision;
    d.tol = opts->tol;
    d.maxiter = opts->maxiter;
    int rc = pycfd_solver_create(&d, &B->solvers[i]);
    if (rc) return bail(rc);
  }
  int rc = opts->precision == PCFD_MIXED ? batch_build<float>(B, descs, structure, dt_ctl, max_steps, u, v, p)
                                         : batch_build<double>(B, descs, structure, dt_ctl, max_steps, u, v, p);
  if (rc) return bail(rc);
  if (cudaHostAlloc((void**)&B->h_any, TK_COUNT * sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&B->h_passes, TK_COUNT * sizeof(long long), cudaHostAllocDefault) != cudaSuccess)
    return bail(fail(PCFD_E_CUDA, "pinned allocation failed"));
  if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(PCFD_E_CUDA, "batch setup failed"));
  *out = B;
  return 0;
}

int pycfd_batch_initialize(pycfd_batch* B, void* stream) {
  if (!B) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  return B->precision == PCFD_MIXED ? b_initialize<float>(B, sm) : b_initialize<double>(B, sm);
}

int pycfd_batch_step(pycfd_batch* B, int steps, int record, void* stream) {
  if (!B || steps < 0) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  if (!record) {
    for (int k = 0; k < steps; ++k) TRY(b_dispatch_step(B, sm));
    return 0;
  }
  if (!B->exec) {
    if (!B->aux) CU(cudaStreamCreateWithFlags(&B->aux, cudaStreamNonBlocking));
    if (!B->aux2) CU(cudaStreamCreateWithFlags(&B->aux2, cudaStreamNonBlocking));
    if (!B->rec) CU(cudaStreamCreateWithFlags(&B->rec, cudaStreamNonBlocking));
    CU(cudaStreamBeginCapture(B->rec, cudaStreamCaptureModeThreadLocal));
    B->capturing = true;
    const long long l0 = g_launches.load();
    int rc = b_dispatch_step(B, B->rec);
    B->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(B->rec, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return fail(PCFD_E_CUDA, "batch step capture failed: %s", cudaGetErrorString(ec));
    const long long rec_total = g_launches.load() - l0;
    // 3 solves per step: each solve's loop bodies counted once while recording
    B->fixed_launches = rec_total - 3 * (B->cg_body_launches + B->ir_body_launches);
    CU(cudaGraphInstantiate(&B->exec, graph, 0));
    B->graph = graph;
  }
  for (int k = 0; k < steps; ++k) CU(cudaGraphLaunch(B->exec, sm));
  return 0;
}

int pycfd_batch_profile(pycfd_batch* B, int kernel_id) {
  if (!B || kernel_id < 0 || kernel_id > 6) return fail(PCFD_E_ARG, "bad arguments");
  return pycfd_profile_kernel(B->mem, kernel_id);
}

int pycfd_batch_profile_read(pycfd_batch* B, double* total_ms, int* launches, void* stream) {
  if (!B) return fail(PCFD_E_ARG, "bad arguments");
  return pycfd_profile_read(B->mem, total_ms, launches, stream);
}

int pycfd_batch_set_loop_cap(pycfd_batch* B, int cap, void* stream) {
  if (!B || cap < 0) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  std::vector<unsigned> c(TK_COUNT, 0u);
  c[TK_CG] = c[TK_IR] = (unsigned)cap;
  CU(cudaMemcpyAsync(B->sh.cap_set, c.data(), TK_COUNT * sizeof(unsigned), cudaMemcpyHostToDevice, sm));
  CU(cudaStreamSynchronize(sm));
  return 0;
}

int pycfd_batch_capped(pycfd_batch* B, int* capped, void* stream) {
  if (!B || !capped) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  int h[TK_COUNT];
  CU(cudaMemcpyAsync(h, B->sh.capped, sizeof h, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  *capped = (h[TK_CG] ? 1 : 0) | (h[TK_IR] ? 2 : 0);
  CU(cudaMemsetAsync(B->sh.capped, 0, sizeof h, sm));
  CU(cudaStreamSynchronize(sm));
  return 0;
}

pycfd_solver* pycfd_batch_problem(pycfd_batch* B, int i) {
  if (!B || i < 0 || i >= B->n) return nullptr;
  return B->solvers[i];
}

int pycfd_batch_status(pycfd_batch* B, int* frozen, int* steps, int* iterations, int* status, double* t,
                       double* dt, void* stream) {
  if (!B) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  if (B->precision == PCFD_MIXED)
    BLAUNCH(k_b_gather<float>, (B->n + 127) / 128, 128, 0, sm, probs_of<float>(B), B->n, B->d_iout, B->d_dout);
  else
    BLAUNCH(k_b_gather<double>, (B->n + 127) / 128, 128, 0, sm, probs_of<double>(B), B->n, B->d_iout, B->d_dout);
  std::vector<int> io((size_t)4 * B->n);
  std::vector<double> dd((size_t)2 * B->n);
  CU(cudaMemcpyAsync(io.data(), B->d_iout, io.size() * sizeof(int), cudaMemcpyDeviceToHost, sm));
  CU(cudaMemcpyAsync(dd.data(), B->d_dout, dd.size() * sizeof(double), cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  for (int k = 0; k < B->n; ++k) {
    if (frozen) frozen[k] = io[4 * k];
    if (steps) steps[k] = io[4 * k + 1];
    if (iterations) iterations[k] = io[4 * k + 2];
    if (status) status[k] = io[4 * k + 3];
    if (t) t[k] = dd[2 * k];
    if (dt) dt[k] = dd[2 * k + 1];
  }
  return 0;
}

// Kernel launches executed on the device since the last call: recorded loop
// bodies times the passes the device ran, plus the fixed part per step.
int pycfd_batch_launches(pycfd_batch* B, int steps, long long* launches, void* stream) {
  if (!B || !launches) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  CU(cudaMemcpyAsync(B->h_passes, B->sh.passes, sizeof(long long) * TK_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  const long long cg = B->h_passes[TK_CG] + B->h_passes[TK_ARM];
  *launches = (long long)steps * B->fixed_launches + cg * B->cg_body_launches +
              B->h_passes[TK_IR] * B->ir_body_launches;
  CU(cudaMemsetAsync(B->sh.passes, 0, sizeof(long long) * TK_COUNT, sm));
  return 0;
}

}  // extern "C"
