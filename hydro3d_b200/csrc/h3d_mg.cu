// Host runtime of the B200 multigrid solver: handle, device layout, V-cycle
// schedule (the reference's K-cycle control flow, mgsolver.for:272-352),
// CUDA-graph capture, the FP64 outer defect correction (newsolv_mg.for) and
// the C ABI declared in include/h3d_mg.h.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "h3d_internal.h"
#include "h3d_kernels.cuh"

using namespace h3d;

namespace {

thread_local std::string g_create_error;

}  // namespace

void h3d::set_call_error(const std::string& msg) { g_create_error = msg; }

namespace {

// Levels with at most this many interior cells relax in one single-CTA launch.
constexpr int64_t kSmallLevelCells = 2048;
// Largest block relaxed by one CTA per visit (a 32^3 block in one CTA is slower
// than the tiled sweep kernels; 16^3 is four cells a thread and colour)
constexpr int64_t kBlockLocalCells = 4096;
constexpr int64_t kTailLevelCells = 2048;  // levels the fused coarse tail (one CTA) takes

struct Halo {
  uint32_t* d_dst = nullptr;
  uint32_t* d_src = nullptr;
  int64_t n = 0;
  bool built = false;
};

// An expression fill on the device (see ExprTable).
struct XFill {
  uint32_t* d_nodes = nullptr;
  uint32_t* d_dst = nullptr;
  uint32_t* d_src = nullptr;
  int64_t nw = 0, nnodes = 0;
  std::vector<int64_t> ds;  // node ranges by depth (host)
  bool built = false;
};

struct Level {
  LevelGeom geom;
  BlkLev* d_bl = nullptr;
  int* d_cta_all = nullptr;  // ghost-inclusive cells
  int ncta_all = 0;
  int* d_cta_int = nullptr;  // interior cells
  int ncta_int = 0;
  int* d_rows_all = nullptr;  // all rows (y, z incl. ghosts)
  int nrows_all = 0;
  int* d_rows_int = nullptr;  // interior rows
  int nrows_int = 0;
  Tile* d_tiles = nullptr;
  int ntiles = 0, tiles_cap = 0;
  int variant = 0, zc = 1;
  double* phi64[2] = {nullptr, nullptr};
  double* rhs64 = nullptr;
  float* phi32[2] = {nullptr, nullptr};
  float* rhs32 = nullptr;
  double *fx64 = nullptr, *fy64 = nullptr, *fz64 = nullptr;
  float *fx32 = nullptr, *fy32 = nullptr, *fz32 = nullptr;
  double* dens = nullptr;
  Halo sweep, faces, exch, bound;
  Halo sweep_push;              // the sweep fill without the faces the register-window sweeps push
  Halo live, live_push;         // the parts of sweep / sweep_push that the next sweep or restriction reads
  bool live_ok = false;         // live fills may stand in for the full fill (FP32 RBGS levels)
  Halo red;                     // red cells next to block faces and the ghosts that show them (k_red_ahead)
  int* d_red_info = nullptr;    // their blocks and wall faces (k_red_ahead)
  bool red_ok = false;          // FP32 sweeps of this level take the red-black order across block faces
  long long* d_push = nullptr;  // per block, six ghost push offsets (kNoPush: none)
  bool push_ok = false;
  CUtensorMap* d_maps = nullptr;  // [ty index][0,1: iterate buffer, 2: rhs][block] tensor maps
  CUtensorMap* d_rmaps = nullptr;  // as the fine level of a restriction: [tyc index][0,1: iterate, 2: rhs][block]
  Tile* d_rtiles = nullptr;       // restriction tiles (this level as the coarse level)
  int rtiles_cap = 0;
  Tile* d_ptiles = nullptr;       // level 1: tiled-defect tiles (kProlongRows rows of one plane, ghosts included)
  int nptiles = 0;
  Tile* d_qtiles = nullptr;       // prolongation tiles (plane pairs 2m, 2m+1 of a block, ghost planes included)
  int nqtiles = 0;
  Tile* d_dtiles = nullptr;       // level 1: z-march defect tiles (defect_march_rows() rows x dzc planes)
  int ndtiles = 0, dzc = 1, dgp = 0;  // dgp: pairs per lane of the z-march defect (0: not usable)
  int* d_dstart = nullptr;        // level 1: first z-march defect tile of each block (nb + 1 entries)
  int* d_pstart = nullptr;        // level 1: first tiled-defect tile of each block (nb + 1 entries)
  bool pvec32 = false, pvec64 = false;  // every block's nx a multiple of 4 (FP32) / 2 (FP64) cells, ny and nz even
  int nrtiles = 0, rvariant = 0, rzc = 1;
  bool tma_ok = false;
  bool f32 = false, var = false;  // iterate precision of the level's smoother; variable coefficients
  int* d_cstart = nullptr;  // small / tail levels: flat interior index of each block's first cell
  bool small = false;       // relaxation runs as one fused single-CTA kernel
  bool blocal = false;      // the sweep fill stays inside every block: a visit is one launch, a CTA per block
  Halo lfill;               // that fill, sorted by block
  int* d_lfstart = nullptr; // its per-block entry ranges (nb + 1)
  bool tailable = false;    // small enough for the fused coarse tail (has d_cstart)
  int cur64 = 0, cur32 = 0;
  bool zero64 = false, zero32 = false;
  Tile* d_ztiles = nullptr;     // FP32 zero-source sweep tiles (launch_rbgs_zero32), or none
  bool use_z32 = true;          // the zero-source kernel beat the tuned sweep's zero mode (autotuner)
  int nztiles = 0, zzc = 1;
  double* seq64 = nullptr;      // line-TDMA scratch a(s) of every cell (mg_itrsch 2)
  float* seq32 = nullptr;
  // local mesh refinement
  bool expr = false;            // the level's fills are expression tables (neighbours of different rdv)
  XFill xs, xe;                 // sweep fill (mgbound + exchangepp), exchangepp alone (built on first use)
  double* xscratch = nullptr;   // node values of the expression fills (FP64 or FP32)
  int64_t xscratch_n = 0;
  int* d_rsame = nullptr;       // blocks past their last level here (restriction into this level is a copy)
  int nrsame = 0, rsame_cells = 0;
  int* d_psame = nullptr;       // blocks whose next coarser level has this level's size (correction is an add)
  int npsame = 0, psame_cells = 0;
  int* d_prows = nullptr;       // prolongation rows of the other blocks (ghost rows included)
  int nprows = 0;
  double sweep_bytes = 0;       // algorithmic bytes of one sweep (FP64 or FP32 by mode)
  double sweep_bytes_zero = 0;  // ... of a sweep from the zero iterate (the iterate is not read)
};

struct CachedGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<int> state_after;
  int64_t kernels = 0;
  std::vector<cudaEvent_t> events;  // profiling pairs recorded inside the graph
  std::vector<double> bytes;         // algorithmic bytes of the sweep each pair brackets
};

}  // namespace

struct h3d_mg {
  int device = 0;
  cudaStream_t st = nullptr;
  h3d_mg_desc desc{};
  std::vector<h3d_block_desc> blocks;
  int L = 1;
  bool mixed = false, var = false;
  std::vector<Level> lev;  // index 1..L
  double* p64[2] = {nullptr, nullptr};
  int pc = 0;
  double* b64 = nullptr;
  double* partials = nullptr;
  int npartials = 0;
  double* d_res = nullptr;
  double* h_res = nullptr;  // pinned, 4 doubles
  bool per_block = false;    // the defect also reduces its partial sums per block (stop_rule 2)
  double* d_resb = nullptr;  // per block {sum r^2, sum b^2, max|r| dV, sum r}
  double* h_resb = nullptr;  // pinned copy of d_resb
  double* d_h3 = nullptr;   // per-block dx,dy,dz
  int* d_err = nullptr;     // set by a device wait that gave up
  double mean_b = 0.0;
  bool coeffs_ready = false;
  std::string last_error;
  // profiling / accounting
  bool profiling = false;
  std::vector<cudaEvent_t> ev_eager;  // events of eager (non-graph) iterations
  int64_t kernels = 0;
  std::map<std::vector<int>, CachedGraph> graphs;
  bool capturing = false;
  bool debug_sync = false;  // H3D_DEBUG_SYNC=1: synchronize and check after every launch
  std::vector<double> history;
  // whole host block arrays staged on the device (0: pressure, 1: rhs) for
  // contiguous host transfers; allocated on first use
  double* stage[2] = {nullptr, nullptr};
  std::vector<size_t> stage_off;
  // fused coarse tail: levels tail_g..L in one single-CTA launch (tail_g = 0: none)
  int tail_g = 0;
  bool lmr = false;  // blocks of different refinement ratio or level count (LMR = 2)
  TailLevel* d_tail_lv = nullptr;
  TailOp* d_tail_ops = nullptr;
  unsigned long long* d_tail_cells = nullptr;  // cell tables of all tail levels
  BlkLev* d_tail_cbl = nullptr;                // compact block tables of the tail levels
  int* d_tail_starts = nullptr;                // cluster tail: per-block fill ranges
  int tail_cluster = 0;                        // cluster tail: CTAs of the cluster (0: single-CTA tail)
  int tail_nlev = 0;
  uint32_t* d_tail_fills = nullptr;            // compact sweep fill tables of the tail levels
  double* d_dense = nullptr;                   // pseudo-inverse of the coarsest level (coarse_direct)
  int dense_n = 0;
  int tail_nops = 0;
  int tail_smem = 0;  // dynamic shared memory of the tail launch
  float omega = 1.f;       // over-relaxation of the FP32 sweeps (desc.omega)
  bool rb_global = false;  // FP32 sweeps take the red-black order across block faces (desc.rb_order)
  std::vector<char> tail_zero32, tail_zero64;  // zero flags of the tail levels after the tail
  // the projection (allocated on first use): face velocities u, v, w and
  // ustar, vstar, wstar in the level-1 layout, and the gather table of their
  // face ghosts (exchange(1..3) after calvel)
  double* vel[3] = {nullptr, nullptr, nullptr};
  double* vstar[3] = {nullptr, nullptr, nullptr};
  uint32_t* d_vdst = nullptr;
  uint32_t* d_vsrc = nullptr;
  int64_t nvfill = 0;
  double* sip[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // SIP factors, res
  double* sip_pp = nullptr;  // the SIP pressure correction (level-1 layout)
  bool proj = false;        // outer iterations end with p += pp, calvel, calmas
  double proj_dtal = 0.0;   // dt*alfapr
  double proj_dt = 1.0;
};

namespace {

int fail(h3d_mg* h, int code, const std::string& msg) {
  if (h) h->last_error = msg;
  else g_create_error = msg;
  return code;
}

#define CU(...)                                                                                   \
  do {                                                                                            \
    cudaError_t _e = (__VA_ARGS__);                                                               \
    if (_e != cudaSuccess)                                                                        \
      return fail(h, _e == cudaErrorMemoryAllocation ? H3D_ERR_OOM : H3D_ERR_CUDA,                \
                  std::string(#__VA_ARGS__).substr(0, 60) + ": " + cudaGetErrorString(_e));       \
  } while (0)

#define TRY(call)                   \
  do {                              \
    int _r = (call);                \
    if (_r != H3D_OK) return _r;    \
  } while (0)

template <typename T>
int dalloc(h3d_mg* h, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) return H3D_OK;
  CU(cudaMalloc((void**)p, n * sizeof(T)));
  // The zero fill must be complete before the caller fills the array: uploads
  // with cudaMemcpy run on the legacy stream, which is not ordered after the
  // solver's non-blocking stream (a late zero fill once wiped freshly
  // uploaded tile lists, and the sweeps then indexed plane -1 of their ring).
  CU(cudaMemsetAsync(*p, 0, n * sizeof(T), h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

// First tile of every block in a tile list whose tiles are grouped by block
// (nb + 1 entries, the last one the tile count), uploaded to *d_start.
int upload_tile_starts(h3d_mg* h, const std::vector<Tile>& tiles, int nb, int** d_start) {
  std::vector<int> st(nb + 1, (int)tiles.size());
  for (int q = (int)tiles.size() - 1; q >= 0; --q) st[tiles[q].b] = q;
  for (int b = nb - 1; b >= 0; --b)
    if (st[b] > st[b + 1]) st[b] = st[b + 1];
  int rc = dalloc(h, d_start, st.size());
  if (rc != H3D_OK) return rc;
  if (cudaMemcpy(*d_start, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(h, H3D_ERR_CUDA, "tile starts");
  return H3D_OK;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

int upload_halo(h3d_mg* h, Halo& H, const std::vector<uint32_t>& d, const std::vector<uint32_t>& s) {
  H.n = (int64_t)d.size();
  if (H.n == 0) return H3D_OK;
  TRY(dalloc(h, &H.d_dst, d.size()));
  TRY(dalloc(h, &H.d_src, s.size()));
  CU(cudaMemcpy(H.d_dst, d.data(), d.size() * 4, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(H.d_src, s.data(), s.size() * 4, cudaMemcpyHostToDevice));
  return H3D_OK;
}

// Builds and uploads the expression form of level g's fill of `kind`.
int upload_xfill(h3d_mg* h, int g, int kind, XFill& X) {
  ExprTable T;
  std::string err;
  const int rc = build_expr_table(h->blocks, g, kind, true, T, &err);
  if (rc != H3D_OK) return fail(h, rc, err);
  Level& V = h->lev[g];
  X.nw = (int64_t)T.dst.size();
  X.nnodes = (int64_t)T.nodes.size() / 9;
  X.ds = T.depth_start;
  if (!T.nodes.empty()) {
    TRY(dalloc(h, &X.d_nodes, T.nodes.size()));
    CU(cudaMemcpy(X.d_nodes, T.nodes.data(), T.nodes.size() * 4, cudaMemcpyHostToDevice));
  }
  if (X.nw > 0) {
    TRY(dalloc(h, &X.d_dst, T.dst.size()));
    TRY(dalloc(h, &X.d_src, T.src.size()));
    CU(cudaMemcpy(X.d_dst, T.dst.data(), T.dst.size() * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(X.d_src, T.src.data(), T.src.size() * 4, cudaMemcpyHostToDevice));
  }
  if (X.nnodes > V.xscratch_n) {
    CU(cudaDeviceSynchronize());
    dfree(V.xscratch);
    V.xscratch = nullptr;
    TRY(dalloc(h, &V.xscratch, (size_t)X.nnodes));
    V.xscratch_n = X.nnodes;
  }
  X.built = true;
  return H3D_OK;
}

// Runs an expression fill: out's ghosts from cur (current values) and old
// (pre-fill values, zero when zero_old).
template <typename T>
cudaError_t run_xfill(const Level& V, const XFill& X, T* out, const T* cur, const T* old, bool zero_old,
                      cudaStream_t st) {
  return launch_expr_fill<T>(X.d_nodes, X.ds.data(), (int)X.ds.size() - 1, X.d_dst, X.d_src, X.nw, out, cur, old,
                             zero_old, reinterpret_cast<T*>(V.xscratch), st);
}

// Uploads a list of block ids; *cells = the largest listed block's cell count
// (interior, or with the ghost layer).
int upload_block_list(h3d_mg* h, const LevelGeom& G, const std::vector<char>& sel, bool ghosts, int** d, int* n,
                      int* cells) {
  std::vector<int> ids;
  long long mc = 0;
  for (size_t b = 0; b < G.bl.size(); ++b)
    if (sel[b]) {
      ids.push_back((int)b);
      const BlkLev& B = G.bl[b];
      mc = std::max(mc, ghosts ? (long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2) : (long long)B.nx * B.ny * B.nz);
    }
  *n = (int)ids.size();
  *cells = (int)mc;
  if (ids.empty()) return H3D_OK;
  TRY(dalloc(h, d, ids.size()));
  CU(cudaMemcpy(*d, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice));
  return H3D_OK;
}

int build_cta_table(h3d_mg* h, const LevelGeom& G, bool interior, int** d_tab, int* ncta) {
  std::vector<int> start(G.bl.size() + 1, 0);
  for (size_t b = 0; b < G.bl.size(); ++b) {
    const BlkLev& B = G.bl[b];
    long long cells = interior ? (long long)B.nx * B.ny * B.nz : (long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2);
    if (cells >= (1LL << 31)) return fail(h, H3D_ERR_BAD_CONFIG, "block too large");
    start[b + 1] = start[b] + (int)((cells + 255) / 256);
  }
  *ncta = start.back();
  TRY(dalloc(h, d_tab, start.size()));
  CU(cudaMemcpy(*d_tab, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
  return H3D_OK;
}

int build_row_table(h3d_mg* h, const LevelGeom& G, bool interior, int** d_tab, int* nrows) {
  std::vector<int> start(G.bl.size() + 1, 0);
  for (size_t b = 0; b < G.bl.size(); ++b) {
    const BlkLev& B = G.bl[b];
    long long rows = interior ? (long long)B.ny * B.nz : (long long)(B.ny + 2) * (B.nz + 2);
    if ((long long)start[b] + rows >= (1LL << 31)) return fail(h, H3D_ERR_BAD_CONFIG, "too many rows");
    start[b + 1] = start[b] + (int)rows;
  }
  *nrows = start.back();
  TRY(dalloc(h, d_tab, start.size()));
  CU(cudaMemcpy(*d_tab, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
  return H3D_OK;
}

// A row-tile smoother variant needs every block's nx even and within its row.
bool variant_fits(const Level& Lv, int variant) {
  TileShape s = tile_shape(variant);
  if (!s.rows) return true;
  if (s.tma && !Lv.tma_ok) return false;
  if (s.tma == 3 && (!Lv.f32 || Lv.var)) return false;
  for (const auto& B : Lv.geom.bl)
    if ((B.nx & 1) || B.nx > s.tx || (s.tma == 3 && (B.nx & 3))) return false;
  return true;
}

// Copies a tile list to its device array, growing the array only when the
// list outgrows it (the autotuners rebuild tile lists many times).
int upload_tiles(h3d_mg* h, Tile** d, int* cap, const std::vector<Tile>& t) {
  if ((int)t.size() > *cap) {
    CU(cudaDeviceSynchronize());
    dfree(*d);
    *d = nullptr;
    *cap = 0;
    TRY(dalloc(h, d, t.size()));
    *cap = (int)t.size();
  }
  CU(cudaMemcpyAsync(*d, t.data(), t.size() * sizeof(Tile), cudaMemcpyHostToDevice, h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int build_tiles(h3d_mg* h, Level& Lv, int variant, int zc) {
  TileShape s = tile_shape(variant);
  std::vector<Tile> t;
  for (size_t b = 0; b < Lv.geom.bl.size(); ++b) {
    const BlkLev& B = Lv.geom.bl[b];
    for (int z0 = 1; z0 <= B.nz; z0 += zc)
      for (int y0 = 1; y0 <= B.ny; y0 += s.ty)
        for (int x0 = 1; x0 <= B.nx; x0 += s.tx) t.push_back(Tile{(int)b, x0, y0, z0});
  }
  TRY(upload_tiles(h, &Lv.d_tiles, &Lv.tiles_cap, t));
  Lv.ntiles = (int)t.size();
  Lv.variant = variant;
  Lv.zc = zc;
  return H3D_OK;
}


// Restriction tiles of (TY rows x all x) x zc planes over every block of the
// coarse geometry G (blocks past their last level restrict by a copy instead).
std::vector<Tile> row_tiles(const LevelGeom& G, int ty, int zc) {
  std::vector<Tile> t;
  for (size_t b = 0; b < G.bl.size(); ++b)
    for (int z0 = 1; !G.clamped[b] && z0 <= G.bl[b].nz; z0 += zc)
      for (int y0 = 1; y0 <= G.bl[b].ny; y0 += ty) t.push_back(Tile{(int)b, 1, y0, z0});
  return t;
}

// z chunk giving at least ~3 CTAs per SM.
int pick_zc(const LevelGeom& G, int ty) {
  int nzm = 1;
  long long xy = 0;
  for (const auto& B : G.bl) {
    nzm = std::max(nzm, B.nz);
    xy += (B.ny + ty - 1) / ty;
  }
  int zc = nzm;
  while (zc > 4 && xy * ((nzm + zc - 1) / zc) < 148 * 3) zc = (zc + 1) / 2;
  return zc;
}

int build_restrict_tiles(h3d_mg* h, Level& C) {
  int nxm = 0;
  for (const auto& B : C.geom.bl) nxm = std::max(nxm, B.nx);
  int v = -1;
  for (int q = 0; q < num_restrict_shapes(); ++q) {
    RestrictShape r = restrict_shape(q);
    if (!r.tma && r.tpr * r.cpx >= nxm) { v = q; break; }
  }
  if (v < 0) return fail(h, H3D_ERR_BAD_CONFIG, "block too wide for the restriction kernels (nx > 512)");
  RestrictShape r = restrict_shape(v);
  int zc = pick_zc(C.geom, r.tyc);
  std::vector<Tile> t = row_tiles(C.geom, r.tyc, zc);
  TRY(upload_tiles(h, &C.d_rtiles, &C.rtiles_cap, t));
  C.nrtiles = (int)t.size();
  C.rvariant = v;
  C.rzc = zc;
  return H3D_OK;
}

// Heuristic tile choice (the autotuner refines it on large levels).
void default_tile(const Level& Lv, int* variant, int* zc) {
  int nxm = 0, nym = 0, nzm = 0;
  long long xy_tiles = 0;
  for (const auto& B : Lv.geom.bl) {
    nxm = std::max(nxm, B.nx);
    nym = std::max(nym, B.ny);
    nzm = std::max(nzm, B.nz);
  }
  int v;
  if (nxm >= 32) v = nym >= 16 ? 0 : 1;
  else if (nxm >= 16) v = 3;
  else if (nxm >= 8) v = nym >= 8 ? 4 : 5;
  else v = 6;
  // whole-row tiles when every block allows them (TMA-staged first)
  const int pref[] = {47, 46, 45, 41, 28, 25, 24, 20, 13, 12, 10, 8, 14, 16};
  for (int cand : pref) {
    TileShape c = tile_shape(cand);
    if (nxm <= c.tx && nxm * 2 > c.tx / 2 && variant_fits(Lv, cand) && nym >= 4) { v = cand; break; }
  }
  TileShape s = tile_shape(v);
  for (const auto& B : Lv.geom.bl) xy_tiles += (long long)((B.nx + s.tx - 1) / s.tx) * ((B.ny + s.ty - 1) / s.ty);
  int z = nzm;
  while (z > 8 && xy_tiles * ((nzm + z - 1) / z) < 148 * 6) z /= 2;
  *variant = v;
  *zc = std::max(1, z);
}


// ------------------------------------------------------------------ executor
// Tensor maps of buffer `buf` for the level's smoother variant (or null).
const CUtensorMap* sweep_maps(const Level& V, int buf) {
  TileShape s = tile_shape(V.variant);
  if (!s.tma || !V.tma_ok) return nullptr;
  int ti = tma_ty_index(s.ty);
  if (ti < 0) return nullptr;
  return V.d_maps + ((size_t)ti * 3 + buf) * V.geom.bl.size();
}

// Restriction tensor maps of fine level F for the coarse level's restriction
// variant: iterate buffer `buf` (rhs = false) or right-hand side, or null.
const CUtensorMap* restrict_maps(const Level& F, int variant, int buf, bool rhs) {
  RestrictShape r = restrict_shape(variant);
  if (!r.tma || !F.d_rmaps) return nullptr;
  int ti = rtma_tyc_index(r.tyc);
  if (ti < 0) return nullptr;
  return F.d_rmaps + ((size_t)ti * 3 + (rhs ? 2 : buf)) * F.geom.bl.size();
}

// Tensor maps of the level's right-hand side (box TY+2 rows), or null.
const CUtensorMap* rhs_maps(const Level& V) {
  TileShape s = tile_shape(V.variant);
  if (s.tma < 2 || !V.tma_ok) return nullptr;
  int ti = tma_ty_index(s.ty);
  if (ti < 0) return nullptr;
  return V.d_maps + ((size_t)ti * 3 + 2) * V.geom.bl.size();
}

// FP32 iterate at level g?  Mixed solves run every level but the coarsest in
// FP32; the coarsest level (the coarse solve) stays FP64.
bool f32_level(const h3d_mg* h, int g) { return h->mixed && !(g == h->L && h->L > 1); }

// The level-1 pressure halo before an FP64 defect: exchange(4) + pbound
// (newsolv_mg.for:51-52), i.e. the face ghosts of the sweep fill; with local
// mesh refinement the sweep's expression fill, in place.
int pressure_halo(h3d_mg* h) {
  Level& V = h->lev[1];
  double* p = h->p64[h->pc];
  if (V.expr) CU(run_xfill<double>(V, V.xs, p, p, p, false, h->st));
  else CU(launch_fill<double>(V.faces.d_dst, V.faces.d_src, V.faces.n, p, p, p, false, h->st));
  return H3D_OK;
}

struct Exec {
  h3d_mg* h;
  std::vector<cudaEvent_t>* prof = nullptr;  // pre-created events for level-1 sweeps
  size_t prof_used = 0;
  std::vector<double> prof_bytes;  // algorithmic bytes of each bracketed sweep

  Level& L(int g) { return h->lev[g]; }

  bool mixed_level(int g) const { return f32_level(h, g); }

  // Debug mode: synchronize after a launch and name the failing operation.
  int chk(const char* what, int g) {
    if (!h->debug_sync) return H3D_OK;
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess)
      return fail(h, H3D_ERR_CUDA, std::string(what) + " (level " + std::to_string(g) + "): " + cudaGetErrorString(e));
    return H3D_OK;
  }

  // Inside stream capture an event must be recorded as an external node to be
  // timed later; outside capture a plain record.
  cudaError_t record(cudaEvent_t e) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t r = cudaStreamIsCapturing(h->st, &cs);
    if (r != cudaSuccess) return r;
    if (cs == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(e, h->st, cudaEventRecordExternal);
    return cudaEventRecord(e, h->st);
  }

  // The fill after a sweep: the dst iterate's ghosts from its interior and
  // the src iterate's ghosts (zero: src is the zero iterate).  Returns the
  // number of kernels it launched.
  template <typename T>
  int sweep_fill(const Level& V, const Halo& H, T* dst, const T* src, bool zero, int64_t* nk) {
    if (V.expr) {
      CU(run_xfill<T>(V, V.xs, dst, dst, src, zero, h->st));
      for (size_t d = 0; d + 1 < V.xs.ds.size(); ++d) *nk += V.xs.ds[d + 1] > V.xs.ds[d];
      *nk += V.xs.nw > 0;
    } else {
      CU(launch_fill<T>(H.d_dst, H.d_src, H.n, dst, dst, src, zero, h->st));
      *nk += H.n > 0;
    }
    return H3D_OK;
  }

  // partial: the next reader of this level is a sweep or a restriction of
  // it, so the fill may leave out the ghosts those never read (live tables)
  int sweep(int g, bool partial = false) {
    Level& V = L(g);
    cudaStream_t st = h->st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // profiling brackets the full level-1 sweeps (3 words a cell); the first
    // sweep from a zero iterate is another kernel with other bytes
    const bool from_zero = mixed_level(g) ? V.zero32 : V.zero64;
    if (h->desc.mg_itrsch == 3 && mixed_level(g) && V.red_ok && !V.zero32) {
      // the red cells next to block faces first: red-black order across blocks
      CU(launch_red_ahead(h->var, V.red.d_dst, V.red.d_src, V.d_red_info, V.red.n, (int)V.geom.bl.size(), V.d_bl,
                          V.phi32[V.cur32], V.rhs32, V.fx32, V.fy32, V.fz32, h->omega, st));
      TRY(chk("red ahead", g));
      h->kernels += 1;
    }
    if (prof && g == 1 && !from_zero && prof_used + 2 <= prof->size()) {
      e0 = (*prof)[prof_used++];
      e1 = (*prof)[prof_used++];
      CU(record(e0));
      prof_bytes.push_back(V.sweep_bytes);
    }
    if (h->desc.mg_itrsch != 3) {  // lexicographic GS or line TDMA: one CTA per block
      const int nb = (int)V.geom.bl.size();
      if (mixed_level(g)) {
        float* src = V.phi32[V.cur32];
        float* dst = V.phi32[1 - V.cur32];
        CU(launch_seq_smoother<float>(h->desc.mg_itrsch, h->var, V.zero32, V.d_bl, nb, src, dst, V.rhs32, V.seq32,
                                      V.fx32, V.fy32, V.fz32, st));
        TRY(chk("sequential sweep fp32", g));
        if (e1) CU(record(e1));
        TRY(sweep_fill<float>(V, V.sweep, dst, src, V.zero32, &h->kernels));
        TRY(chk("fill fp32", g));
        V.cur32 = 1 - V.cur32;
        V.zero32 = false;
      } else {
        double* src = V.phi64[V.cur64];
        double* dst = V.phi64[1 - V.cur64];
        CU(launch_seq_smoother<double>(h->desc.mg_itrsch, h->var, V.zero64, V.d_bl, nb, src, dst, V.rhs64, V.seq64,
                                       V.fx64, V.fy64, V.fz64, st));
        TRY(chk("sequential sweep fp64", g));
        if (e1) CU(record(e1));
        TRY(sweep_fill<double>(V, V.sweep, dst, src, V.zero64, &h->kernels));
        TRY(chk("fill fp64", g));
        V.cur64 = 1 - V.cur64;
        V.zero64 = false;
      }
      h->kernels += 1;
      return H3D_OK;
    }
    if (mixed_level(g) && V.zero32 && V.d_ztiles && V.use_z32) {  // first sweep from a zero iterate: a stencil on rhs
      float* src = V.phi32[V.cur32];
      float* dst = V.phi32[1 - V.cur32];
      const bool push = V.push_ok;
      CU(launch_rbgs_zero32(V.d_bl, V.d_ztiles, V.nztiles, V.zzc, V.rhs32, dst, push ? V.d_push : nullptr, h->omega,
                            st));
      TRY(chk("zero-source sweep fp32", g));
      if (e1) CU(record(e1));
      const Halo& fill = partial && V.live_ok ? (push ? V.live_push : V.live) : (push ? V.sweep_push : V.sweep);
      TRY(sweep_fill<float>(V, fill, dst, src, true, &h->kernels));
      TRY(chk("fill fp32", g));
      V.cur32 = 1 - V.cur32;
      V.zero32 = false;
      h->kernels += 1;
      return H3D_OK;
    }
    if (mixed_level(g)) {
      float* src = V.phi32[V.cur32];
      float* dst = V.phi32[1 - V.cur32];
      const bool push = V.push_ok && rbgs_pushes(V.variant, h->var, true);
      CU(launch_rbgs<float>(V.variant, h->var, V.zero32, V.d_bl, V.d_tiles, V.ntiles, V.zc, sweep_maps(V, V.cur32),
                            rhs_maps(V), h->d_err, src, dst, V.rhs32,
                            V.fx32, V.fy32, V.fz32, push ? V.d_push : nullptr, h->omega, st));
      TRY(chk("sweep fp32", g));
      if (e1) CU(record(e1));
      const Halo& fill = partial && V.live_ok ? (push ? V.live_push : V.live) : (push ? V.sweep_push : V.sweep);
      TRY(sweep_fill<float>(V, fill, dst, src, V.zero32, &h->kernels));
      TRY(chk("fill fp32", g));
      V.cur32 = 1 - V.cur32;
      V.zero32 = false;
    } else {
      double* src = V.phi64[V.cur64];
      double* dst = V.phi64[1 - V.cur64];
      CU(launch_rbgs<double>(V.variant, h->var, V.zero64, V.d_bl, V.d_tiles, V.ntiles, V.zc, sweep_maps(V, V.cur64),
                             rhs_maps(V), h->d_err, src, dst, V.rhs64,
                             V.fx64, V.fy64, V.fz64, nullptr, 1.f, st));
      TRY(chk("sweep fp64", g));
      if (e1) CU(record(e1));
      TRY(sweep_fill<double>(V, V.sweep, dst, src, V.zero64, &h->kernels));
      TRY(chk("fill fp64", g));
      V.cur64 = 1 - V.cur64;
      V.zero64 = false;
    }
    h->kernels += 1;
    return H3D_OK;
  }

  // live_next: the visit's next reader of level g is a restriction from it or
  // another sweep of it (they read the live ghosts only)
  int relax(int g, int it, bool live_next = false) {
    Level& V = L(g);
    if (it > 0 && V.small && g > 1 && h->desc.mg_itrsch == 3) {  // all sweeps and fills of this visit in one launch
      const int nb = (int)V.geom.bl.size();
      if (mixed_level(g)) {
        CU(launch_relax_small<float>(h->var, V.d_bl, V.d_cstart, nb, V.phi32[V.cur32], V.rhs32, V.fx32, V.fy32,
                                     V.fz32, V.sweep.d_dst, V.sweep.d_src, (int)V.sweep.n, it, V.zero32,
                                     V.geom.n_elems, h->omega, h->rb_global, h->st));
        V.zero32 = false;
      } else {
        CU(launch_relax_small<double>(h->var, V.d_bl, V.d_cstart, nb, V.phi64[V.cur64], V.rhs64, V.fx64, V.fy64,
                                      V.fz64, V.sweep.d_dst, V.sweep.d_src, (int)V.sweep.n, it, V.zero64,
                                      V.geom.n_elems, 1.f, false, h->st));
        V.zero64 = false;
      }
      TRY(chk("relax small", g));
      h->kernels += 1;
      return H3D_OK;
    }
    if (it > 0 && V.blocal && g > 1 && h->desc.mg_itrsch == 3) {  // a visit in one launch, a CTA per block
      const int nb = (int)V.geom.bl.size();
      if (mixed_level(g)) {
        CU(launch_relax_blocks<float>(h->var, V.d_bl, nb, V.d_lfstart, V.phi32[V.cur32], V.rhs32, V.fx32, V.fy32,
                                      V.fz32, V.lfill.d_dst, V.lfill.d_src, it, V.zero32, h->omega, h->st));
        V.zero32 = false;
      } else {
        CU(launch_relax_blocks<double>(h->var, V.d_bl, nb, V.d_lfstart, V.phi64[V.cur64], V.rhs64, V.fx64, V.fy64,
                                       V.fz64, V.lfill.d_dst, V.lfill.d_src, it, V.zero64, 1.f, h->st));
        V.zero64 = false;
      }
      TRY(chk("relax blocks", g));
      h->kernels += 1;
      return H3D_OK;
    }
    for (int q = 0; q < it; ++q) TRY(sweep(g, live_next || q + 1 < it));
    return H3D_OK;
  }

  // coarse rhs of level gc from the fine level gc-1 (mgrestr(gc))
  int restrict_to(int gc) {
    Level& F = L(gc - 1);
    Level& C = L(gc);
    if (mixed_level(gc - 1)) {
      // the coarsest level of a mixed solve keeps an FP32 rhs too (converted after)
      CU(launch_restrict_tile<float>(C.rvariant, h->var, F.zero32, F.d_bl, C.d_bl, C.d_rtiles, C.nrtiles, C.rzc,
                                     F.phi32[F.cur32], F.rhs32, C.rhs32, F.fx32, F.fy32, F.fz32,
                                     restrict_maps(F, C.rvariant, F.cur32, false),
                                     restrict_maps(F, C.rvariant, 0, true), h->d_err, h->st));
      TRY(chk("restrict fp32", gc));
      if (C.nrsame > 0) {
        CU(launch_restrict_same<float>(F.zero32, F.d_bl, C.d_bl, C.d_rsame, C.nrsame, C.rsame_cells,
                                       F.phi32[F.cur32], F.rhs32, C.rhs32, h->st));
        h->kernels += 1;
      }
      C.zero32 = true;
      if (!mixed_level(gc)) {  // coarsest level solved in FP64
        CU(launch_convert_f2d(C.rhs32, C.rhs64, C.geom.n_elems, h->st));
        TRY(chk("convert rhs f2d", gc));
        C.zero64 = true;
        h->kernels += 1;
      }
    } else {
      CU(launch_restrict_tile<double>(C.rvariant, h->var, F.zero64, F.d_bl, C.d_bl, C.d_rtiles, C.nrtiles, C.rzc,
                                      F.phi64[F.cur64], F.rhs64, C.rhs64, F.fx64, F.fy64, F.fz64,
                                      restrict_maps(F, C.rvariant, F.cur64, false),
                                      restrict_maps(F, C.rvariant, 0, true), h->d_err, h->st));
      TRY(chk("restrict fp64", gc));
      if (C.nrsame > 0) {
        CU(launch_restrict_same<double>(F.zero64, F.d_bl, C.d_bl, C.d_rsame, C.nrsame, C.rsame_cells,
                                        F.phi64[F.cur64], F.rhs64, C.rhs64, h->st));
        h->kernels += 1;
      }
      C.zero64 = true;
    }
    h->kernels += 1;
    return H3D_OK;
  }

  // mgcorr(gf): correction from level gf+1 into level gf, with mgbound fused
  int correct(int gf) {
    Level& F = L(gf);
    Level& C = L(gf + 1);
    RowTab ct{F.d_prows ? F.d_prows : F.d_rows_all, (int)F.geom.bl.size(), F.d_prows ? F.nprows : F.nrows_all};
    if (mixed_level(gf)) {
      const float* pc;
      if (mixed_level(gf + 1)) {
        if (C.zero32) TRY(materialize_zero32(gf + 1));
        pc = C.phi32[C.cur32];
      } else {  // coarsest solved in FP64: bring its iterate to FP32
        if (C.zero64) TRY(materialize_zero64(gf + 1));
        CU(launch_convert_d2f(C.phi64[C.cur64], C.phi32[C.cur32], C.geom.n_elems, h->st));
        TRY(chk("convert phi d2f", gf + 1));
        h->kernels += 1;
        pc = C.phi32[C.cur32];
      }
      if (F.pvec32)
        CU(launch_prolong_vec<float>(F.zero32, F.d_bl, C.d_bl, F.d_qtiles, F.nqtiles, pc, F.phi32[F.cur32],
                                     F.phi32[1 - F.cur32], h->st));
      else
        CU(launch_prolong<float>(F.zero32, F.d_bl, C.d_bl, ct, pc, F.phi32[F.cur32], F.phi32[1 - F.cur32], h->st));
      if (F.npsame > 0) {
        CU(launch_prolong_same<float>(F.zero32, F.d_bl, C.d_bl, F.d_psame, F.npsame, F.psame_cells, pc,
                                      F.phi32[F.cur32], F.phi32[1 - F.cur32], h->st));
        h->kernels += 1;
      }
      TRY(chk("prolong fp32", gf));
      F.cur32 = 1 - F.cur32;
      F.zero32 = false;
    } else {
      if (C.zero64) TRY(materialize_zero64(gf + 1));
      if (F.pvec64)
        CU(launch_prolong_vec<double>(F.zero64, F.d_bl, C.d_bl, F.d_qtiles, F.nqtiles, C.phi64[C.cur64],
                                      F.phi64[F.cur64], F.phi64[1 - F.cur64], h->st));
      else
        CU(launch_prolong<double>(F.zero64, F.d_bl, C.d_bl, ct, C.phi64[C.cur64], F.phi64[F.cur64],
                                  F.phi64[1 - F.cur64], h->st));
      if (F.npsame > 0) {
        CU(launch_prolong_same<double>(F.zero64, F.d_bl, C.d_bl, F.d_psame, F.npsame, F.psame_cells,
                                       C.phi64[C.cur64], F.phi64[F.cur64], F.phi64[1 - F.cur64], h->st));
        h->kernels += 1;
      }
      TRY(chk("prolong fp64", gf));
      F.cur64 = 1 - F.cur64;
      F.zero64 = false;
    }
    h->kernels += 1;
    return H3D_OK;
  }

  int materialize_zero64(int g) {
    Level& V = L(g);
    CU(cudaMemsetAsync(V.phi64[V.cur64], 0, V.geom.n_elems * sizeof(double), h->st));
    V.zero64 = false;
    return H3D_OK;
  }
  int materialize_zero32(int g) {
    Level& V = L(g);
    CU(cudaMemsetAsync(V.phi32[V.cur32], 0, V.geom.n_elems * sizeof(float), h->st));
    V.zero32 = false;
    return H3D_OK;
  }

  // mgkcyc control flow (mgsolver.for:272-352) with kcycle = 1.
  // the fused coarse tail (levels tail_g..L), entered right after the
  // restriction into level tail_g
  int tail() {
    const int g0 = h->tail_g;
    unsigned mask = 0;
    for (int g = g0; g <= h->L; ++g) {
      const Level& V = L(g);
      mask |= (unsigned)(V.cur32 & 1) << (2 * (g - g0));
      mask |= (unsigned)(V.cur64 & 1) << (2 * (g - g0) + 1);
    }
    if (h->tail_cluster)
      CU(launch_coarse_cluster(h->tail_cluster, h->d_tail_lv, h->tail_nlev, h->d_tail_ops, h->tail_nops, mask,
                               h->tail_smem, h->st));
    else
      CU(launch_coarse_tail(h->d_tail_lv, h->d_tail_ops, h->tail_nops, mask, h->tail_smem, h->st));
    TRY(chk("coarse tail", g0));
    for (int g = g0; g <= h->L; ++g) {
      L(g).zero32 = h->tail_zero32[g - g0] != 0;
      L(g).zero64 = h->tail_zero64[g - g0] != 0;
    }
    h->kernels += 1;
    return H3D_OK;
  }

  // more: another V-cycle follows on the same level-1 iterate (its first reader
  // is a sweep), so the last level-1 sweep may leave out the unread ghosts
  int vcycle(bool more = false) {
    const int Lv = h->L;
    const int irestr = h->desc.irestr, iproln = h->desc.iproln;
    const int csw = h->desc.coarse_sweeps;
    auto relax_at = [&](int g, int it, bool coarsest_first, bool live_next) -> int {
      if (g == Lv && Lv > 1 && csw > 0) return coarsest_first ? relax(g, csw) : H3D_OK;
      return relax(g, it, live_next);
    };
    if (Lv == 1) {
      if (csw > 0) return relax(1, csw);
      TRY(relax(1, irestr));
      return relax(1, iproln);
    }
    TRY(relax(1, irestr, true));
    TRY(restrict_to(2));
    int kount[kMaxLevels + 2] = {0};
    int g = 2, nrel = irestr;
    for (;;) {
      if (g == 1) break;
      if (g == h->tail_g && kount[g] == 0) {  // levels g..L in one launch, up to g's post-relaxation
        TRY(tail());
        TRY(correct(g - 1));
        g -= 1;
        nrel = iproln;
        continue;
      }
      kount[g] += 1;
      TRY(relax_at(g, nrel, true, kount[g] != 2 && g < Lv));
      if (kount[g] == 2) {
        TRY(correct(g - 1));
        kount[g] = 0;
        g -= 1;
        nrel = iproln;
      } else if (g < Lv) {
        TRY(restrict_to(g + 1));
        g += 1;
        nrel = irestr;
      } else {
        TRY(relax_at(g, iproln, false, false));
        TRY(correct(g - 1));
        nrel = iproln;
        g = Lv - 1;
      }
    }
    return relax(1, iproln, more);
  }

  // FP64 defect on the resident p/b: e = level-1 iterate (or none).
  int defect(bool with_e) {
    Level& V = L(1);
    RowTab ct{V.d_rows_all, (int)V.geom.bl.size(), V.nrows_all};
    // rmax = max |r| dV (press.for:61-63): sup already carries dV (L_LSM);
    // otherwise each block's own cell volume (-1), which differs with refinement
    double rscale = h->var ? 1.0 : -1.0;
    const double* fx = h->var ? V.fx64 : nullptr;
    const double* fy = h->var ? V.fy64 : nullptr;
    const double* fz = h->var ? V.fz64 : nullptr;
    double* pin = h->p64[h->pc];
    double* pout = h->p64[1 - h->pc];
    // the z-march and tiled kernels need constant coefficients and nx even
    const bool march = V.dgp > 0 && !h->var;
    const bool tiled = !march && V.d_ptiles && V.pvec64 && !h->var;
    const int ngrid = march ? V.ndtiles : tiled ? V.nptiles : defect_grid(ct.nrows);
    if (h->mixed) {
      const float* e = nullptr;
      if (with_e) {
        if (V.zero32) TRY(materialize_zero32(1));
        e = V.phi32[V.cur32];
      }
      if (march)
        CU(launch_defect_march<float, float>(V.dgp, V.d_bl, V.d_dtiles, V.ndtiles, V.dzc, pin, e, pout, h->b64,
                                             V.rhs32, h->mean_b, rscale, h->partials, h->st));
      else if (tiled)
        CU(launch_defect_vec<float, float>(V.d_bl, V.d_ptiles, V.nptiles, pin, e, pout, h->b64, V.rhs32, h->mean_b,
                                           rscale, h->partials, ngrid, h->st));
      else
        CU(launch_defect<float, float>(h->var, V.d_bl, ct, pin, e, pout, h->b64, V.rhs32, h->mean_b, rscale, fx, fy,
                                       fz, h->partials, h->st));
    } else {
      const double* e = nullptr;
      if (with_e) {
        if (V.zero64) TRY(materialize_zero64(1));
        e = V.phi64[V.cur64];
      }
      if (march)
        CU(launch_defect_march<double, double>(V.dgp, V.d_bl, V.d_dtiles, V.ndtiles, V.dzc, pin, e, pout, h->b64,
                                               V.rhs64, h->mean_b, rscale, h->partials, h->st));
      else if (tiled)
        CU(launch_defect_vec<double, double>(V.d_bl, V.d_ptiles, V.nptiles, pin, e, pout, h->b64, V.rhs64,
                                             h->mean_b, rscale, h->partials, ngrid, h->st));
      else
        CU(launch_defect<double, double>(h->var, V.d_bl, ct, pin, e, pout, h->b64, V.rhs64, h->mean_b, rscale, fx,
                                         fy, fz, h->partials, h->st));
    }
    TRY(chk("defect", 1));
    if (with_e) h->pc = 1 - h->pc;
    CU(launch_reduce4(h->partials, ngrid, h->d_res, h->st));
    TRY(chk("reduce", 1));
    CU(cudaMemcpyAsync(h->h_res, h->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    h->kernels += 2;
    if (h->per_block && h->blocks.size() > 1) {
      // the march and tiled defects write one partial per tile, tiles grouped by block
      const int* start = march ? V.d_dstart : tiled ? V.d_pstart : nullptr;
      if (!start) return fail(h, H3D_ERR_BAD_CONFIG, "per-block stop rule: the defect of this layout has no per-block partial sums");
      const int nb = (int)h->blocks.size();
      CU(launch_reduce4_blocks(h->partials, start, nb, h->d_resb, h->st));
      TRY(chk("reduce per block", 1));
      CU(cudaMemcpyAsync(h->h_resb, h->d_resb, 4 * sizeof(double) * nb, cudaMemcpyDeviceToHost, h->st));
      h->kernels += 1;
    }
    return H3D_OK;
  }

  // One outer iteration: V-cycle(s) on the current defect, then p += e and
  // the new defect (the projection: p += e, exchange(4) + pbound, calvel,
  // calmas).
  int iteration(int inner) {
    Level& V = L(1);
    if (h->mixed) V.zero32 = true;
    else V.zero64 = true;
    for (int q = 0; q < inner; ++q) TRY(vcycle(q + 1 < inner));
    if (h->proj) {
      TRY(proj_update());
      return vel_defect();
    }
    if (h->lmr) {
      // p += e, then the pressure halo of p itself (exchange(4) + pbound,
      // newsolv_mg.for:39-52): with refinement the ghosts are averages and
      // extrapolations, so the ghosts of p + e are not those of p plus e's
      RowTab ra{V.d_rows_all, (int)V.geom.bl.size(), V.nrows_all};
      double* p = h->p64[h->pc];
      if (h->mixed) {
        if (V.zero32) TRY(materialize_zero32(1));
        CU(launch_padd<float>(V.d_bl, ra, p, V.phi32[V.cur32], h->st));
      } else {
        if (V.zero64) TRY(materialize_zero64(1));
        CU(launch_padd<double>(V.d_bl, ra, p, V.phi64[V.cur64], h->st));
      }
      TRY(chk("p update", 1));
      TRY(pressure_halo(h));
      TRY(chk("pressure halo", 1));
      h->kernels += 2;
      return defect(false);
    }
    return defect(true);
  }

  // newsolv_mg.for:39-52: p = p + (pp - ppref) over the block and its ghost
  // layer, then exchange(4) + pbound (the face ghosts of the interior rows).
  int proj_update() {
    Level& V = L(1);
    RowTab ra{V.d_rows_all, (int)V.geom.bl.size(), V.nrows_all};
    double* p = h->p64[h->pc];
    if (h->mixed) {
      if (V.zero32) TRY(materialize_zero32(1));
      CU(launch_padd<float>(V.d_bl, ra, p, V.phi32[V.cur32], h->st));
    } else {
      if (V.zero64) TRY(materialize_zero64(1));
      CU(launch_padd<double>(V.d_bl, ra, p, V.phi64[V.cur64], h->st));
    }
    TRY(chk("p update", 1));
    CU(launch_fill<double>(V.faces.d_dst, V.faces.d_src, V.faces.n, p, p, p, false, h->st));
    TRY(chk("pressure halo", 1));
    h->kernels += 2;
    return H3D_OK;
  }

  // calvel with its exchange(1..3), then calmas into the level-1 right-hand
  // side and the FP64 su (newsolv_mg.for:54-55); the sums reach h_res.
  int vel_defect() {
    Level& V = L(1);
    RowTab ri{V.d_rows_int, (int)V.geom.bl.size(), V.nrows_int};
    CU(launch_calvel(h->var, V.d_bl, ri, h->d_h3, h->p64[h->pc], V.dens, h->vstar[0], h->vstar[1], h->vstar[2],
                     h->vel[0], h->vel[1], h->vel[2], h->proj_dtal, h->st));
    TRY(chk("calvel", 1));
    CU(launch_gather3(h->d_vdst, h->d_vsrc, h->nvfill, h->vel[0], h->vel[1], h->vel[2], h->st));
    TRY(chk("velocity exchange", 1));
    int np = 0;
    if (h->mixed)
      CU(launch_calmas<float>(h->var, V.d_bl, ri, h->d_h3, h->vel[0], h->vel[1], h->vel[2], h->proj_dt, h->b64,
                              V.rhs32, h->partials, &np, h->st));
    else
      CU(launch_calmas<double>(h->var, V.d_bl, ri, h->d_h3, h->vel[0], h->vel[1], h->vel[2], h->proj_dt, h->b64,
                               V.rhs64, h->partials, &np, h->st));
    TRY(chk("calmas", 1));
    CU(launch_reduce4(h->partials, np, h->d_res, h->st));
    TRY(chk("reduce", 1));
    CU(cudaMemcpyAsync(h->h_res, h->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    h->kernels += (h->nvfill > 0) ? 4 : 3;
    return H3D_OK;
  }
};

std::vector<int> state_key(h3d_mg* h, int tag) {
  std::vector<int> k;
  k.push_back(tag);
  k.push_back(h->pc);
  for (int g = 1; g <= h->L; ++g) {
    k.push_back(h->lev[g].cur64);
    k.push_back(h->lev[g].cur32);
    k.push_back(h->lev[g].zero64);
    k.push_back(h->lev[g].zero32);
  }
  return k;
}

void set_state(h3d_mg* h, const std::vector<int>& k) {
  size_t q = 1;
  h->pc = k[q++];
  for (int g = 1; g <= h->L; ++g) {
    h->lev[g].cur64 = k[q++];
    h->lev[g].cur32 = k[q++];
    h->lev[g].zero64 = k[q++];
    h->lev[g].zero32 = k[q++];
  }
}

int accumulate_events(h3d_mg* h, const std::vector<cudaEvent_t>& ev, const std::vector<double>& bytes, double* ms,
                      int64_t* n, double* nbytes) {
  for (size_t q = 0; q + 1 < ev.size(); q += 2) {
    float t = 0;
    CU(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
    *ms += t;
    *n += 1;
    if (q / 2 < bytes.size()) *nbytes += bytes[q / 2];
  }
  return H3D_OK;
}

// Events needed to bracket the level-1 sweeps of one outer iteration.
size_t events_per_iteration(const h3d_mg* h, int inner) {
  int sweeps1 = h->desc.irestr + h->desc.iproln;
  if (h->L == 1 && h->desc.coarse_sweeps > 0) sweeps1 = h->desc.coarse_sweeps;
  return 2 * (size_t)inner * (size_t)sweeps1;
}

int make_events(h3d_mg* h, std::vector<cudaEvent_t>& ev, size_t n) {
  while (ev.size() < n) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    ev.push_back(e);
  }
  return H3D_OK;
}

// Runs one outer iteration through a cached CUDA graph (captured on first use
// for the current buffer state) or eagerly.
int run_iteration(h3d_mg* h, int inner, double* prof_ms, int64_t* prof_n, double* prof_bytes) {
  const size_t nev = h->profiling ? events_per_iteration(h, inner) : 0;
  if (!h->desc.use_graph) {
    TRY(make_events(h, h->ev_eager, nev));
    Exec ex{h, h->profiling ? &h->ev_eager : nullptr};
    TRY(ex.iteration(inner));
    CU(cudaStreamSynchronize(h->st));
    std::vector<cudaEvent_t> used(h->ev_eager.begin(), h->ev_eager.begin() + ex.prof_used);
    return accumulate_events(h, used, ex.prof_bytes, prof_ms, prof_n, prof_bytes);
  }
  std::vector<int> key =
      state_key(h, inner * 8 + (h->profiling ? 1 : 0) + (h->per_block ? 2 : 0) + (h->proj ? 4 : 0));
  auto it = h->graphs.find(key);
  if (it == h->graphs.end()) {
    CachedGraph cg;
    TRY(make_events(h, cg.events, nev));
    Exec ex{h, h->profiling ? &cg.events : nullptr};
    int64_t k0 = h->kernels;
    CU(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = ex.iteration(inner);
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
    if (rc != H3D_OK) {
      if (graph) cudaGraphDestroy(graph);
      for (auto e : cg.events) cudaEventDestroy(e);
      return rc;
    }
    if (ce != cudaSuccess) return fail(h, H3D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&cg.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(h, H3D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    cg.kernels = h->kernels - k0;
    h->kernels = k0;
    cg.events.resize(ex.prof_used);
    cg.bytes = ex.prof_bytes;
    cg.state_after = state_key(h, key[0]);
    it = h->graphs.emplace(key, cg).first;
    set_state(h, key);
  }
  CU(cudaGraphLaunch(it->second.exec, h->st));
  h->kernels += it->second.kernels;
  set_state(h, it->second.state_after);
  CU(cudaStreamSynchronize(h->st));
  return accumulate_events(h, it->second.events, it->second.bytes, prof_ms, prof_n, prof_bytes);
}

bool is_all_neumann(const h3d_mg* h) {
  for (const auto& d : h->blocks)
    for (int f = 0; f < 6; ++f)
      if (d.bc[f] == 5) return false;
  return true;
}

int copy_field_3d(h3d_mg* h, bool to_device, double* dev_base, const BlkLev& B, double* host,
                  const h3d_block_desc& d, bool with_ghosts) {
  // canonical (x,y,z) <-> host (pl-1+x, pl-1+y, pl-1+z)
  const int g0 = with_ghosts ? 0 : 1;
  const int ex = with_ghosts ? B.nx + 2 : B.nx, ey = with_ghosts ? B.ny + 2 : B.ny, ez = with_ghosts ? B.nz + 2 : B.nz;
  cudaMemcpy3DParms p{};
  cudaPitchedPtr dptr = make_cudaPitchedPtr(dev_base + B.off, (size_t)B.sx * 8, B.nx + 2, B.ny + 2);
  cudaPitchedPtr hptr = make_cudaPitchedPtr(host, (size_t)d.ttc[0] * 8, d.ttc[0], d.ttc[1]);
  cudaPos dpos = make_cudaPos((size_t)g0 * 8, g0, g0);
  cudaPos hpos = make_cudaPos((size_t)(d.pl - 1 + g0) * 8, d.pl - 1 + g0, d.pl - 1 + g0);
  if (to_device) {
    p.srcPtr = hptr; p.srcPos = hpos; p.dstPtr = dptr; p.dstPos = dpos; p.kind = cudaMemcpyHostToDevice;
  } else {
    p.srcPtr = dptr; p.srcPos = dpos; p.dstPtr = hptr; p.dstPos = hpos; p.kind = cudaMemcpyDeviceToHost;
  }
  p.extent = make_cudaExtent((size_t)ex * 8, ey, ez);
  CU(cudaMemcpy3DAsync(&p, h->st));
  return H3D_OK;
}

int check_block_host_dims(h3d_mg* h, const h3d_block_desc& d) {
  if (d.pl < 1) return fail(h, H3D_ERR_ARG, "pl must be >= 1");
  for (int a = 0; a < 3; ++a)
    if (d.ttc[a] < d.n[a] + 2 * d.pl) return fail(h, H3D_ERR_ARG, "ttc smaller than n + 2*pl");
  return H3D_OK;
}

// Host <-> device through the staging buffers: the whole host block array
// moves with one contiguous copy, a kernel moves the canonical region between
// staging and the padded layout.  stage_out writes back whole host planes, so
// it is only used in calls that staged the same host array in (the planes'
// other cells then round-trip unchanged).
int ensure_stage(h3d_mg* h) {
  if (h->stage[0]) return H3D_OK;
  size_t n = 0;
  h->stage_off.clear();
  for (const auto& d : h->blocks) {
    h->stage_off.push_back(n);
    n += (size_t)d.ttc[0] * d.ttc[1] * d.ttc[2];
  }
  TRY(dalloc(h, &h->stage[0], n));
  TRY(dalloc(h, &h->stage[1], n));
  return H3D_OK;
}

int stage_in(h3d_mg* h, int f, int ib, const double* host, double* dev_level, bool with_ghosts) {
  const h3d_block_desc& d = h->blocks[ib];
  TRY(check_block_host_dims(h, d));
  TRY(ensure_stage(h));
  const BlkLev& B = h->lev[1].geom.bl[ib];
  double* stg = h->stage[f] + h->stage_off[ib];
  CU(cudaMemcpyAsync(stg, host, (size_t)d.ttc[0] * d.ttc[1] * d.ttc[2] * sizeof(double), cudaMemcpyHostToDevice,
                     h->st));
  const int g0 = with_ghosts ? 0 : 1, e = with_ghosts ? 2 : 0;
  CU(launch_stage(true, stg, d.ttc[0], d.ttc[1], d.pl, g0, B.nx + e, B.ny + e, B.nz + e, dev_level + B.off, B.sx,
                  B.sxy, h->st));
  return H3D_OK;
}

int stage_out(h3d_mg* h, int f, int ib, double* host, double* dev_level, bool with_ghosts) {
  const h3d_block_desc& d = h->blocks[ib];
  const BlkLev& B = h->lev[1].geom.bl[ib];
  double* stg = h->stage[f] + h->stage_off[ib];
  const int g0 = with_ghosts ? 0 : 1, e = with_ghosts ? 2 : 0;
  CU(launch_stage(false, stg, d.ttc[0], d.ttc[1], d.pl, g0, B.nx + e, B.ny + e, B.nz + e, dev_level + B.off, B.sx,
                  B.sxy, h->st));
  const size_t plane = (size_t)d.ttc[0] * d.ttc[1];
  const size_t z0 = (size_t)(d.pl - 1 + g0), nzp = (size_t)(B.nz + e);
  CU(cudaMemcpyAsync(host + z0 * plane, stg + z0 * plane, nzp * plane * sizeof(double), cudaMemcpyDeviceToHost,
                     h->st));
  return H3D_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor maps of both iterate buffers and of the right-hand side of level g
// for every TMA box height: origin kXOff elements before x = 0, dims
// (nx+2+kXOff, ny+2, nz+2), strides (sx, sxy) elements, box (BX, TY+4 or
// TY+2, 1), out-of-bounds rows read as zero.  Levels whose row width exceeds
// one box (BX > 256) or with an odd nx keep the plain-load smoothers.
int build_tensor_maps(h3d_mg* h, int g) {
  Level& V = h->lev[g];
  const bool f32 = f32_level(h, g);
  const int es = f32 ? 4 : 8, vec = 16 / es;
  for (const auto& B : V.geom.bl) {
    int bx = (B.nx + 2 + kXOff + vec - 1) / vec * vec;
    if ((B.nx & 1) || bx > 256) return H3D_OK;
  }
  auto enc = encode_fn();
  if (!enc) return H3D_OK;
  const size_t nb = V.geom.bl.size();
  std::vector<CUtensorMap> maps((size_t)kNumTmaTy * 3 * nb);
  const int tys[kNumTmaTy] = {4, 8, 16, 32, 15};
  for (int ti = 0; ti < kNumTmaTy; ++ti)
    for (int buf = 0; buf < 3; ++buf)
      for (size_t b = 0; b < nb; ++b) {
        const BlkLev& B = V.geom.bl[b];
        // the box starts kXOff elements before x = 0, on the row's 16-byte boundary
        const long long o = B.off - kXOff;
        void* base = buf == 2 ? (f32 ? (void*)(V.rhs32 + o) : (void*)(V.rhs64 + o))
                              : (f32 ? (void*)(V.phi32[buf] + o) : (void*)(V.phi64[buf] + o));
        cuuint64_t dims[3] = {(cuuint64_t)B.nx + 2 + kXOff, (cuuint64_t)B.ny + 2, (cuuint64_t)B.nz + 2};
        cuuint64_t strides[2] = {(cuuint64_t)B.sx * es, (cuuint64_t)B.sxy * es};
        // iterate: rows y0-2 .. y0+TY+1; right-hand side: rows y0-1 .. y0+TY
        cuuint32_t box[3] = {(cuuint32_t)((B.nx + 2 + kXOff + vec - 1) / vec * vec),
                             (cuuint32_t)(tys[ti] + (buf == 2 ? 2 : 4)), 1};
        cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = enc(&maps[((size_t)ti * 3 + buf) * nb + b], f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                                     : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return H3D_OK;  // keep the plain-load smoothers
      }
  TRY(dalloc(h, &V.d_maps, maps.size()));
  CU(cudaMemcpy(V.d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  // restriction from this level: iterate boxes of 2*TYC+2 fine rows, rhs boxes of 2*TYC rows
  std::vector<CUtensorMap> rm((size_t)kNumRTmaTyc * 3 * nb);
  const int tycs[kNumRTmaTyc] = {4, 8};
  for (int ti = 0; ti < kNumRTmaTyc; ++ti)
    for (int buf = 0; buf < 3; ++buf)
      for (size_t b = 0; b < nb; ++b) {
        const BlkLev& B = V.geom.bl[b];
        const long long o = B.off - kXOff;
        void* base = buf == 2 ? (f32 ? (void*)(V.rhs32 + o) : (void*)(V.rhs64 + o))
                              : (f32 ? (void*)(V.phi32[buf] + o) : (void*)(V.phi64[buf] + o));
        cuuint64_t dims[3] = {(cuuint64_t)B.nx + 2 + kXOff, (cuuint64_t)B.ny + 2, (cuuint64_t)B.nz + 2};
        cuuint64_t strides[2] = {(cuuint64_t)B.sx * es, (cuuint64_t)B.sxy * es};
        cuuint32_t box[3] = {(cuuint32_t)((B.nx + 2 + kXOff + vec - 1) / vec * vec),
                             (cuuint32_t)(2 * tycs[ti] + (buf == 2 ? 0 : 2)), 1};
        cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = enc(&rm[((size_t)ti * 3 + buf) * nb + b],
                         f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims,
                         strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
          V.tma_ok = true;  // smoother maps are fine; restriction keeps the plain-load kernels
          return H3D_OK;
        }
      }
  TRY(dalloc(h, &V.d_rmaps, rm.size()));
  CU(cudaMemcpy(V.d_rmaps, rm.data(), rm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  V.tma_ok = true;
  return H3D_OK;
}

int check_device_error(h3d_mg* h) {
  int e = 0;
  CU(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CU(cudaMemset(h->d_err, 0, sizeof(int)));
    return fail(h, H3D_ERR_TIMEOUT, "a bounded device wait gave up (TMA copy did not complete)");
  }
  return H3D_OK;
}

// Evicts the L2 (126 MB) before a timed autotuning launch, as in a solve,
// where the kernels in between touch other arrays: overwrites the outer
// solver's spare pressure buffer (one FP64 level-1 field), which holds no
// state between solves.
int flush_l2(h3d_mg* h) {
  const size_t n = (size_t)h->lev[1].geom.n_elems * sizeof(double);
  if (n >= ((size_t)160 << 20)) CU(cudaMemsetAsync(h->p64[1 - h->pc], 0, n, h->st));
  return H3D_OK;
}

int autotune_level(h3d_mg* h, int g) {
  Level& V = h->lev[g];
  int best_v = V.variant, best_z = V.zc;
  if (V.geom.n_interior < 64 || (V.small && g > 1)) return H3D_OK;  // tiny or fused levels: no sweep kernels
  int nzm = 0, nxm = 0, nym = 0;
  for (const auto& B : V.geom.bl) { nzm = std::max(nzm, B.nz); nxm = std::max(nxm, B.nx); nym = std::max(nym, B.ny); }
  cudaEvent_t a, b;
  CU(cudaEventCreate(&a));
  CU(cudaEventCreate(&b));
  float best = 1e30f, best_tz = 1e30f;
  const bool f32 = f32_level(h, g);
  for (int v = 0; v < num_tile_shapes(); ++v) {
    TileShape s = tile_shape(v);
    if (!variant_fits(V, v)) continue;
    if (s.rows ? (s.tx >= 4 * nxm) : (s.tx > 2 * nxm || s.ty > 2 * nym || (s.tx < 8 && nxm >= 32))) continue;
    for (int zc : {1, 2, 4, 8, 16, 32, 64, 128, 256}) {
      if (zc > nzm || (zc < 8 && V.geom.n_interior >= (1 << 20))) continue;
      TRY(build_tiles(h, V, v, zc));
      // a cycle runs sweeps from a non-zero and from the zero iterate: fastest
      // repetition of each, weighted by how often a solve runs them (level 1
      // of a mixed solve: 5 to 1 with two inner cycles; otherwise 2 to 1)
      float tn = 1e30f, tz = 1e30f;
      for (int rep = 0; rep < 12; ++rep) {
        const bool zero = rep >= 6;
        TRY(flush_l2(h));
        CU(cudaEventRecord(a, h->st));
        const long long* push = (f32 && V.push_ok && rbgs_pushes(v, h->var, true)) ? V.d_push : nullptr;
        if (f32) CU(launch_rbgs<float>(v, h->var, zero, V.d_bl, V.d_tiles, V.ntiles, zc, sweep_maps(V, V.cur32),
                                       rhs_maps(V), h->d_err, V.phi32[V.cur32],
                                       V.phi32[1 - V.cur32], V.rhs32, V.fx32, V.fy32, V.fz32, push, h->omega,
                                       h->st));
        else CU(launch_rbgs<double>(v, h->var, zero, V.d_bl, V.d_tiles, V.ntiles, zc, sweep_maps(V, V.cur64),
                                    rhs_maps(V), h->d_err, V.phi64[V.cur64],
                                    V.phi64[1 - V.cur64], V.rhs64, V.fx64, V.fy64, V.fz64, nullptr, 1.f, h->st));
        CU(cudaEventRecord(b, h->st));
        {
          cudaError_t e = cudaEventSynchronize(b);
          int werr = 0;
          if (e == cudaSuccess) e = cudaMemcpy(&werr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost);
          if (e != cudaSuccess || werr)
            return fail(h, e != cudaSuccess ? H3D_ERR_CUDA : H3D_ERR_TIMEOUT,
                        "smoother autotuning (level " + std::to_string(g) + ", variant " + std::to_string(v) +
                            ", z-chunk " + std::to_string(zc) + "): " +
                            (e != cudaSuccess ? cudaGetErrorString(e) : "a bounded device wait gave up"));
        }
        float t;
        CU(cudaEventElapsedTime(&t, a, b));
        if (rep % 6 > 0) (zero ? tz : tn) = std::min(zero ? tz : tn, t);
      }
      const float tot = tn * ((g == 1 && h->mixed) ? 5.f : 2.f) + tz;
      if (tot < best) { best = tot; best_v = v; best_z = zc; best_tz = tz; }
    }
  }
  TRY(build_tiles(h, V, best_v, best_z));
  // the first sweep from a zero iterate: the zero-source stencil kernel or the
  // chosen sweep's zero mode, whichever is faster on this level
  if (f32 && !h->var && V.d_ztiles && V.nztiles > 0) {
    const long long* push = (V.push_ok && rbgs_pushes(V.variant, h->var, true)) ? V.d_push : nullptr;
    float tz32 = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
      TRY(flush_l2(h));
      CU(cudaEventRecord(a, h->st));
      CU(launch_rbgs_zero32(V.d_bl, V.d_ztiles, V.nztiles, V.zzc, V.rhs32, V.phi32[1 - V.cur32], push, h->omega,
                            h->st));
      CU(cudaEventRecord(b, h->st));
      CU(cudaEventSynchronize(b));
      float t;
      CU(cudaEventElapsedTime(&t, a, b));
      if (rep > 0) tz32 = std::min(tz32, t);
    }
    V.use_z32 = tz32 < best_tz;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return H3D_OK;
}

// Times every restriction variant and coarse z-chunk that fits the level
// pair (fine level gc-1 with at least 64 cells) and keeps the fastest.
int autotune_restrict(h3d_mg* h, int gc) {
  Level& F = h->lev[gc - 1];
  Level& C = h->lev[gc];
  if (F.geom.n_interior < 64) return H3D_OK;
  int nxm = 0, nzm = 0;
  for (const auto& B : C.geom.bl) { nxm = std::max(nxm, B.nx); nzm = std::max(nzm, B.nz); }
  const bool f32 = F.f32;
  cudaEvent_t a, b;
  CU(cudaEventCreate(&a));
  CU(cudaEventCreate(&b));
  float best = 1e30f;
  int best_v = C.rvariant, best_z = C.rzc;
  for (int v = 0; v < num_restrict_shapes(); ++v) {
    RestrictShape r = restrict_shape(v);
    if (r.tpr * r.cpx < nxm) continue;
    if (r.tma && (!F.tma_ok || !F.d_rmaps)) continue;
    for (int zc : {1, 2, 4, 8, 16, 32, 64}) {
      if (zc > nzm) continue;
      std::vector<Tile> t = row_tiles(C.geom, r.tyc, zc);
      TRY(upload_tiles(h, &C.d_rtiles, &C.rtiles_cap, t));
      C.nrtiles = (int)t.size();
      float tot = 1e30f;  // fastest of the timed repetitions
      for (int rep = 0; rep < 6; ++rep) {
        TRY(flush_l2(h));
        CU(cudaEventRecord(a, h->st));
        if (f32)
          CU(launch_restrict_tile<float>(v, h->var, false, F.d_bl, C.d_bl, C.d_rtiles, C.nrtiles, zc,
                                         F.phi32[F.cur32], F.rhs32, C.rhs32, F.fx32, F.fy32, F.fz32,
                                         restrict_maps(F, v, F.cur32, false), restrict_maps(F, v, 0, true), h->d_err,
                                         h->st));
        else
          CU(launch_restrict_tile<double>(v, h->var, false, F.d_bl, C.d_bl, C.d_rtiles, C.nrtiles, zc,
                                          F.phi64[F.cur64], F.rhs64, C.rhs64, F.fx64, F.fy64, F.fz64,
                                          restrict_maps(F, v, F.cur64, false), restrict_maps(F, v, 0, true),
                                          h->d_err, h->st));
        CU(cudaEventRecord(b, h->st));
        cudaError_t e = cudaEventSynchronize(b);
        int werr = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&werr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess || werr)
          return fail(h, e != cudaSuccess ? H3D_ERR_CUDA : H3D_ERR_TIMEOUT,
                      "restriction autotuning (level " + std::to_string(gc) + ", variant " + std::to_string(v) +
                          ", z-chunk " + std::to_string(zc) + "): " +
                          (e != cudaSuccess ? cudaGetErrorString(e) : "a bounded device wait gave up"));
        float ms;
        CU(cudaEventElapsedTime(&ms, a, b));
        if (rep > 0) tot = std::min(tot, ms);
      }
      if (tot < best) { best = tot; best_v = v; best_z = zc; }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  RestrictShape r = restrict_shape(best_v);
  std::vector<Tile> t = row_tiles(C.geom, r.tyc, best_z);
  TRY(upload_tiles(h, &C.d_rtiles, &C.rtiles_cap, t));
  C.nrtiles = (int)t.size();
  C.rvariant = best_v;
  C.rzc = best_z;
  return H3D_OK;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

const char* h3d_mg_strerror(int code) {
  switch (code) {
    case H3D_OK: return "ok";
    case H3D_ERR_BAD_CONFIG: return "configuration not supported";
    case H3D_ERR_CUDA: return "CUDA error";
    case H3D_ERR_NOT_CONVERGED: return "not converged";
    case H3D_ERR_DIVERGED: return "diverged";
    case H3D_ERR_TIMEOUT: return "device wait timed out";
    case H3D_ERR_NO_DEVICE: return "no suitable CUDA device";
    case H3D_ERR_ARG: return "bad argument";
    case H3D_ERR_OOM: return "out of device memory";
    case H3D_ERR_INTERNAL: return "internal error";
    default: return "unknown error";
  }
}

const char* h3d_mg_last_error(const h3d_mg* h) { return h ? h->last_error.c_str() : g_create_error.c_str(); }

int h3d_topology(int32_t nblocks, const int32_t* ext, const int32_t* bc, const double* hh, int32_t ngrid,
                 h3d_block_desc* out) {
  // read_infodom (alloc_dom.for:524-1200) on integer extents.
  if (nblocks <= 0 || !ext || !bc || !hh || !out) return H3D_ERR_ARG;
  auto E = [&](int b, int q) { return ext[6 * b + q]; };
  int lo[3] = {E(0, 0), E(0, 2), E(0, 4)}, hi[3] = {E(0, 1), E(0, 3), E(0, 5)};
  for (int b = 1; b < nblocks; ++b)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], E(b, 2 * a));
      hi[a] = std::max(hi[a], E(b, 2 * a + 1));
    }
  for (int a = 0; a < nblocks; ++a) {
    h3d_block_desc& d = out[a];
    std::memset(&d, 0, sizeof(d));
    for (int q = 0; q < 3; ++q) {
      d.n[q] = E(a, 2 * q + 1) - E(a, 2 * q);
      d.origin[q] = E(a, 2 * q);
      d.ttc[q] = d.n[q] + 2;
      d.h[q] = hh[q];
      if (d.n[q] <= 0) return H3D_ERR_ARG;
    }
    d.pl = 1;
    d.ngrid = ngrid;
    d.rdiv = 1;
    for (int q = 0; q < 6; ++q) { d.bc[q] = bc[q]; d.nb_face[q] = -1; d.nb_periodic[q] = -1; }
    for (int q = 0; q < 8; ++q) d.nb_corner[q] = -1;
    for (int q = 0; q < 12; ++q) d.nb_edge[q] = -1;
    // side s of axis q: 0 = low face of a touches high face of b; 1 = high touches low
    auto touch = [&](int b, int q, int s) {
      return s == 0 ? E(a, 2 * q) == E(b, 2 * q + 1) : E(a, 2 * q + 1) == E(b, 2 * q);
    };
    auto same = [&](int b, int q) { return E(a, 2 * q) == E(b, 2 * q) && E(a, 2 * q + 1) == E(b, 2 * q + 1); };
    int cnt[26] = {0};
    for (int b = 0; b < nblocks; ++b) {
      if (b == a) continue;
      for (int q = 0; q < 3; ++q)
        for (int s = 0; s < 2; ++s) {
          int o1 = (q + 1) % 3, o2 = (q + 2) % 3;
          if (touch(b, q, s) && same(b, o1) && same(b, o2)) { d.nb_face[2 * q + s] = b; cnt[2 * q + s]++; }
        }
      // corners: prev #1..4 at z-, next #1..4 at z+ (x,y sides per alloc_dom.for:700-810)
      static const int csx[8] = {0, 0, 1, 1, 1, 1, 0, 0}, csy[8] = {0, 1, 1, 0, 1, 0, 0, 1},
                       csz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
      for (int c = 0; c < 8; ++c)
        if (touch(b, 0, csx[c]) && touch(b, 1, csy[c]) && touch(b, 2, csz[c])) { d.nb_corner[c] = b; cnt[6 + c]++; }
      // edges: (axis pair, sides, running axis) per alloc_dom.for:824-1040
      static const int ea1[12] = {0, 1, 0, 1, 0, 0, 0, 1, 0, 1, 0, 0};
      static const int es1[12] = {0, 1, 1, 0, 0, 0, 1, 0, 0, 1, 1, 1};
      static const int ea2[12] = {2, 2, 2, 2, 1, 1, 2, 2, 2, 2, 1, 1};
      static const int es2[12] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 0};
      static const int erun[12] = {1, 0, 1, 0, 2, 2, 1, 0, 1, 0, 2, 2};
      for (int e = 0; e < 12; ++e)
        if (touch(b, ea1[e], es1[e]) && touch(b, ea2[e], es2[e]) && same(b, erun[e])) {
          d.nb_edge[e] = b;
          cnt[14 + e]++;
        }
    }
    for (int q = 0; q < 26; ++q)
      if (cnt[q] > 1) return H3D_ERR_BAD_CONFIG;
  }
  // periodic partners (alloc_dom.for:1042-1200)
  for (int a = 0; a < nblocks; ++a) {
    h3d_block_desc& d = out[a];
    for (int b = 0; b < nblocks; ++b) {
      if (b == a) continue;
      for (int q = 0; q < 3; ++q) {
        int o1 = (q + 1) % 3, o2 = (q + 2) % 3;
        bool so = E(a, 2 * o1) == E(b, 2 * o1) && E(a, 2 * o1 + 1) == E(b, 2 * o1 + 1) &&
                  E(a, 2 * o2) == E(b, 2 * o2) && E(a, 2 * o2 + 1) == E(b, 2 * o2 + 1);
        if (!so) continue;
        if (bc[2 * q] == 5 && d.nb_face[2 * q] < 0 && E(b, 2 * q + 1) == hi[q]) d.nb_periodic[2 * q] = b;
        if (bc[2 * q + 1] == 5 && d.nb_face[2 * q + 1] < 0 && E(b, 2 * q) == lo[q]) d.nb_periodic[2 * q + 1] = b;
      }
    }
  }
  return H3D_OK;
}

// The live part of a sweep fill: face ghosts of faces that are not physical
// walls.  A sweep and the residual of a restriction read a cell's six face
// neighbours only, with a zero coefficient across a wall (mgsolver.for:186-205),
// so edge, corner and wall ghosts written after a sweep whose next reader is
// one of those are never read.  Prolongation from the level and the outer
// defect read the whole ghost shell: the last sweep before them keeps the full
// fill.  Returns false (no live tables) unless every source is a current
// interior cell, so that one full fill after any number of live ones leaves
// the same ghost shell as full fills throughout.
// Block and (x, y, z) of element gi of a level (blocks in increasing offset).
bool locate_cell(const LevelGeom& G, long long gi, int* b, int* x, int* y, int* z) {
  int lo = 0, hi = (int)G.bl.size() - 1, q = -1;
  while (lo <= hi) {  // last block whose offset is at most gi
    const int mid = (lo + hi) / 2;
    if (G.bl[mid].off <= gi) { q = mid; lo = mid + 1; }
    else hi = mid - 1;
  }
  if (q < 0) return false;
  const BlkLev& B = G.bl[q];
  const long long l = gi - B.off;
  if (l >= B.sxy * (B.nz + 2)) return false;
  *z = (int)(l / B.sxy);
  *y = (int)((l % B.sxy) / B.sx);
  *x = (int)(l % B.sx);
  *b = q;
  return *x <= B.nx + 1;
}

bool live_entries(const LevelGeom& G, const std::vector<uint32_t>& d, const std::vector<uint32_t>& s,
                  std::vector<uint32_t>* ld, std::vector<uint32_t>* ls) {
  auto locate = [&](uint32_t gi, int* b, int* x, int* y, int* z) { return locate_cell(G, gi, b, x, y, z); };
  ld->clear();
  ls->clear();
  for (size_t e = 0; e < d.size(); ++e) {
    int bs, xs, ys, zs, bd, x, y, z;
    if ((s[e] & kOldFlag) || !locate(s[e] & kIdxMask, &bs, &xs, &ys, &zs)) return false;
    const BlkLev& S = G.bl[bs];
    if (xs < 1 || xs > S.nx || ys < 1 || ys > S.ny || zs < 1 || zs > S.nz) return false;
    if (!locate(d[e], &bd, &x, &y, &z)) return false;
    const BlkLev& D = G.bl[bd];
    const bool ox = x == 0 || x == D.nx + 1, oy = y == 0 || y == D.ny + 1, oz = z == 0 || z == D.nz + 1;
    if (ox + oy + oz != 1) continue;  // interior (none in a sweep fill), edge or corner ghost
    const int f = ox ? (x == 0 ? 0 : 1) : oy ? (y == 0 ? 2 : 3) : (z == 0 ? 4 : 5);
    if (D.phys & (1 << f)) continue;  // a wall: zero coefficient
    ld->push_back(d[e]);
    ls->push_back(s[e]);
  }
  return true;
}

// The red cells among the sources of a level's live fill (every block of even
// size, so that colours agree across block faces), for k_red_ahead.
int build_red_ahead(h3d_mg* h, Level& V, const std::vector<uint32_t>& ld, const std::vector<uint32_t>& ls) {
  const auto& G = V.geom;
  for (const auto& B : G.bl)
    if ((B.nx | B.ny | B.nz) & 1) return H3D_OK;
  std::vector<uint32_t> rd, rs;
  std::vector<int> rb;
  for (size_t e = 0; e < ld.size(); ++e) {
    int q, x, y, z;
    if (!locate_cell(G, ls[e] & kIdxMask, &q, &x, &y, &z)) return H3D_OK;  // (sources are interior cells)
    const BlkLev& B = G.bl[q];
    if ((x + y + z) & 1) {  // red
      const int m = B.phys & ((x == 1 ? 1 : 0) | (x == B.nx ? 2 : 0) | (y == 1 ? 4 : 0) | (y == B.ny ? 8 : 0) |
                              (z == 1 ? 16 : 0) | (z == B.nz ? 32 : 0));
      rd.push_back(ld[e]);
      rs.push_back(ls[e]);
      rb.push_back(q | (m << 16));
    }
  }
  if (rd.empty() || G.bl.size() > 0xffff) return H3D_OK;
  TRY(upload_halo(h, V.red, rd, rs));
  TRY(dalloc(h, &V.d_red_info, rb.size()));
  CU(cudaMemcpy(V.d_red_info, rb.data(), rb.size() * sizeof(int), cudaMemcpyHostToDevice));
  V.red_ok = true;
  return H3D_OK;
}

int build_live(h3d_mg* h, Level& V, const std::vector<uint32_t>& d, const std::vector<uint32_t>& s) {
  std::vector<uint32_t> ld, ls;
  V.live_ok = live_entries(V.geom, d, s, &ld, &ls);
  if (V.live_ok) TRY(upload_halo(h, V.live, ld, ls));
  if (V.live_ok && h->mixed && h->desc.mg_itrsch == 3 && h->rb_global) TRY(build_red_ahead(h, V, ld, ls));
  return H3D_OK;
}

// Ghost pushes of a level: a whole face of ghost cells of block bd whose
// sweep-fill sources are, cell for cell, the adjacent face of interior cells
// of one block bs (same pitches) is written by bs's register-window sweep
// (an element offset from each source cell to its ghost), and left out of
// the fill table.  Faces with any other source pattern stay in the table.
int build_push(h3d_mg* h, Level& V, const std::vector<uint32_t>& d, const std::vector<uint32_t>& s) {
  const auto& G = V.geom;
  const int nb = (int)G.bl.size();
  auto locate = [&](uint32_t gi, int* b, int* x, int* y, int* z) -> bool {
    for (int q = 0; q < nb; ++q) {
      const BlkLev& B = G.bl[q];
      const long long lo = B.off, hi = B.off + B.sxy * (B.nz + 2);
      if ((long long)gi < lo || (long long)gi >= hi) continue;
      const long long l = (long long)gi - lo;
      *z = (int)(l / B.sxy);
      *y = (int)((l % B.sxy) / B.sx);
      *x = (int)(l % B.sx);
      *b = q;
      return *x <= B.nx + 1;
    }
    return false;
  };
  struct Face { int bs = -2, side = -1, cnt = 0; bool bad = false; };
  std::vector<Face> face(nb * 6);
  std::vector<int> efac(d.size(), -1);
  for (size_t e = 0; e < d.size(); ++e) {
    int bd, x, y, z;
    if (!locate(d[e], &bd, &x, &y, &z)) continue;
    const BlkLev& D = G.bl[bd];
    const int out = (x == 0 || x == D.nx + 1) + (y == 0 || y == D.ny + 1) + (z == 0 || z == D.nz + 1);
    if (out != 1) continue;
    const int f = x == 0 ? 0 : x == D.nx + 1 ? 1 : y == 0 ? 2 : y == D.ny + 1 ? 3 : z == 0 ? 4 : 5;
    Face& F = face[bd * 6 + f];
    efac[e] = bd * 6 + f;
    F.cnt++;
    int bs, xs, ys, zs;
    if ((s[e] & kOldFlag) || !locate(s[e] & kIdxMask, &bs, &xs, &ys, &zs)) { F.bad = true; continue; }
    const BlkLev& S = G.bl[bs];
    int side = -1;
    if (f < 2) {
      if (ys == y && zs == z && S.nx > 1) side = xs == 1 ? 0 : xs == S.nx ? 1 : -1;
    } else if (f < 4) {
      if (xs == x && zs == z && S.ny > 1) side = ys == 1 ? 2 : ys == S.ny ? 3 : -1;
    } else {
      if (xs == x && ys == y && S.nz > 1) side = zs == 1 ? 4 : zs == S.nz ? 5 : -1;
    }
    if (side < 0) { F.bad = true; continue; }
    if (F.bs == -2) { F.bs = bs; F.side = side; }
    else if (F.bs != bs || F.side != side) F.bad = true;
  }
  std::vector<long long> delta(nb * 6, kNoPush);
  std::vector<char> pushed(nb * 6, 0);
  for (int bd = 0; bd < nb; ++bd)
    for (int f = 0; f < 6; ++f) {
      const Face& F = face[bd * 6 + f];
      const BlkLev& D = G.bl[bd];
      const long long area = f < 2 ? (long long)D.ny * D.nz : f < 4 ? (long long)D.nx * D.nz : (long long)D.nx * D.ny;
      if (F.bad || F.bs < 0 || F.cnt != area) continue;
      const BlkLev& S = G.bl[F.bs];
      if (S.sx != D.sx || S.sxy != D.sxy) continue;
      long long& dl = delta[F.bs * 6 + F.side];
      if (dl != kNoPush) continue;  // the source face already feeds another ghost face
      const long long base = D.off - S.off;
      const int g = (f & 1) ? (f < 2 ? D.nx + 1 : f < 4 ? D.ny + 1 : D.nz + 1) : 0;  // ghost coordinate
      switch (F.side) {
        case 0: dl = base + (g - 1); break;
        case 1: dl = base + (g - S.nx); break;
        case 2: dl = base + (long long)(g - 1) * D.sx; break;
        case 3: dl = base + (long long)(g - S.ny) * D.sx; break;
        case 4: dl = base + (long long)(g - 1) * D.sxy; break;
        default: dl = base + (long long)(g - S.nz) * D.sxy; break;
      }
      pushed[bd * 6 + f] = 1;
    }
  std::vector<uint32_t> rd, rs;
  for (size_t e = 0; e < d.size(); ++e)
    if (efac[e] < 0 || !pushed[efac[e]]) {
      rd.push_back(d[e]);
      rs.push_back(s[e]);
    }
  TRY(dalloc(h, &V.d_push, delta.size()));
  CU(cudaMemcpy(V.d_push, delta.data(), delta.size() * sizeof(long long), cudaMemcpyHostToDevice));
  TRY(upload_halo(h, V.sweep_push, rd, rs));
  if (V.live_ok) {  // the live part of the pushed fill (a subset of a valid table)
    std::vector<uint32_t> ld, ls;
    if (!live_entries(V.geom, rd, rs, &ld, &ls)) return fail(h, H3D_ERR_INTERNAL, "live push table");
    TRY(upload_halo(h, V.live_push, ld, ls));
  }
  V.push_ok = true;
  return H3D_OK;
}

// The fused coarse tail: the deepest run of levels g..L (g >= 2, at least two
// levels, constant coefficients) whose arrays all fit the shared arena of one
// CTA.  Its op program replays, from the moment the restriction into level g
// has run, exactly what Exec::vcycle would launch for those levels
// (relaxations with their zero-iterate flags, restrictions, the FP64
// coarsest level's conversions, corrections), up to the post-relaxation of
// level g; the correction into level g-1 stays outside.  The program starts
// by loading level g's rhs and ends by storing every tail level.
namespace {
struct TailPlan {
  std::vector<int> s_phi32, s_rhs32, s_phi64, s_rhs64;  // arena offsets per tail level
  int scratch = 0, bytes = 0;
};
bool plan_tail(const h3d_mg* h, int g0, TailPlan* P) {
  auto al = [](int v) { return (v + 15) & ~15; };
  int at = 0, scratch = 0;
  for (int q = g0; q <= h->L; ++q) {
    const Level& V = h->lev[q];
    int npad = 0, nint = (int)V.geom.n_interior;
    for (const auto& B : V.geom.bl) npad += (B.nx + 2) * (B.ny + 2) * (B.nz + 2);
    const bool f32 = f32_level(h, q), f64 = !f32 || (h->mixed && q == h->L);
    const bool use32 = h->mixed;
    int p32 = -1, r32 = -1, p64 = -1, r64 = -1;
    if (use32) { p32 = at; at = al(at + npad * 4); r32 = at; at = al(at + nint * 4); }
    if (f64) { p64 = at; at = al(at + npad * 8); r64 = at; at = al(at + nint * 8); }
    P->s_phi32.push_back(p32);
    P->s_rhs32.push_back(r32);
    P->s_phi64.push_back(p64);
    P->s_rhs64.push_back(r64);
    if (q < h->L) scratch = std::max(scratch, (npad - nint) * (f32 ? 4 : 8));
  }
  P->scratch = at;
  P->bytes = al(at + scratch) + 128;
  return P->bytes <= kTailSmemBytes;
}
}  // namespace

// The op program of a tail from level g0 (see build_tail); z32 / z64 return
// the zero flags of every level after it.
void emit_tail_ops(const h3d_mg* h, int g0, int scratch, std::vector<TailOp>& ops, std::vector<char>& z32,
                   std::vector<char>& z64, bool dense = false) {
  const int Lv = h->L;
  const int irestr = h->desc.irestr, iproln = h->desc.iproln, csw = h->desc.coarse_sweeps;
  auto ti = [&](int g) { return g - g0; };
  z32.assign(Lv + 2, 0);
  z64.assign(Lv + 2, 0);
  if (f32_level(h, g0)) z32[g0] = 1;
  else z64[g0] = 1;
  ops.clear();
  auto op = [&](int kind, bool f64, int fine, int coarse, int sweeps, int zero) {
    ops.push_back(TailOp{kind, f64 ? 1 : 0, ti(fine), ti(coarse), sweeps, zero});
  };
  op(kTailLoadRhs, !f32_level(h, g0), g0, g0, 0, 0);
  auto relax = [&](int g, int it) {
    if (it <= 0) return;
    const bool f32 = f32_level(h, g);
    char& z = f32 ? z32[g] : z64[g];
    op(kTailRelax, !f32, g, g, it, z);
    z = 0;
  };
  auto relax_at = [&](int g, int it, bool first) {
    if (g == Lv && Lv > 1 && csw > 0) {
      if (first && dense && !f32_level(h, g)) {  // the coarsest level solved by its pseudo-inverse
        op(kTailDense, true, g, g, 0, z64[g]);
        z64[g] = 0;
      } else if (first) {
        relax(g, csw);
      }
      return;
    }
    relax(g, it);
  };
  auto restrict_to = [&](int gc) {
    const bool f32 = f32_level(h, gc - 1);
    op(kTailRestrict, !f32, gc - 1, gc, 0, f32 ? z32[gc - 1] : z64[gc - 1]);
    if (f32) {
      z32[gc] = 1;
      if (!f32_level(h, gc)) {
        op(kTailRhsF2D, true, gc, gc, 0, 0);
        z64[gc] = 1;
      }
    } else {
      z64[gc] = 1;
    }
  };
  auto zero_fill = [&](int g, bool f64) { op(kTailRelax, f64, g, g, 0, 1); };
  auto correct = [&](int gf) {
    const int gc = gf + 1;
    if (f32_level(h, gf)) {
      if (f32_level(h, gc)) {
        if (z32[gc]) { zero_fill(gc, false); z32[gc] = 0; }
      } else {
        if (z64[gc]) { zero_fill(gc, true); z64[gc] = 0; }
        op(kTailPhiD2F, false, gc, gc, 0, 0);
      }
      op(kTailProlong, false, gf, gc, scratch, z32[gf]);
      z32[gf] = 0;
    } else {
      if (z64[gc]) { zero_fill(gc, true); z64[gc] = 0; }
      op(kTailProlong, true, gf, gc, scratch, z64[gf]);
      z64[gf] = 0;
    }
  };
  // the loop of Exec::vcycle from the first visit of level g0 on
  std::vector<int> kount(Lv + 2, 0);
  int g = g0, nrel = irestr;
  for (;;) {
    kount[g] += 1;
    relax_at(g, nrel, true);
    if (kount[g] == 2) {
      if (g == g0) break;
      correct(g - 1);
      kount[g] = 0;
      g -= 1;
      nrel = iproln;
    } else if (g < Lv) {
      restrict_to(g + 1);
      g += 1;
      nrel = irestr;
    } else {
      relax_at(g, iproln, false);
      correct(g - 1);
      nrel = iproln;
      g = Lv - 1;
      if (g < g0) break;
    }
  }
  for (int q = g0; q <= Lv; ++q) op(kTailStore, false, q, q, 0, 0);
}

int build_tail(h3d_mg* h) {
  const int Lv = h->L;
  if (h->var || h->lmr || h->desc.mg_itrsch != 3) return H3D_OK;  // the fused tail relaxes by red-black GS
  int g0 = Lv + 1;
  TailPlan plan;
  for (int g = Lv; g >= 2; --g) {
    TailPlan P;
    if (!h->lev[g].tailable || !plan_tail(h, g, &P)) break;
    g0 = g;
    plan = P;
  }
  if (g0 > Lv - 1 || Lv - g0 + 1 > kTailMaxLevels) return H3D_OK;  // fewer than two tail levels
  std::vector<TailOp> ops;
  std::vector<char> z32, z64;
  emit_tail_ops(h, g0, plan.scratch, ops, z32, z64);
  // compact layouts, cell tables and fill tables
  std::vector<unsigned long long> cells;
  std::vector<uint32_t> fills;
  std::vector<BlkLev> cbl;
  struct At { size_t cells, ghosts, cbl, fdst, fsrc; int nint, nred, nghost, npad, nfill; };
  std::vector<At> at;
  for (int q = g0; q <= Lv; ++q) {
    const Level& V = h->lev[q];
    At a{};
    a.cbl = cbl.size();
    std::vector<long long> pbase, rbase;
    long long pb = 0, rb = 0;
    for (const auto& B : V.geom.bl) {
      if (B.nx + 1 > 255 || B.ny + 1 > 255 || B.nz + 1 > 255) return H3D_OK;
      BlkLev c = B;
      c.off = pb;
      c.sx = B.nx + 2;
      c.sxy = (long long)(B.nx + 2) * (B.ny + 2);
      c.pad = (int)rb;
      cbl.push_back(c);
      pbase.push_back(pb);
      rbase.push_back(rb);
      pb += c.sxy * (B.nz + 2);
      rb += (long long)B.nx * B.ny * B.nz;
    }
    if (pb >= (1LL << 24)) return H3D_OK;
    std::vector<unsigned long long> red, black, ghost;
    for (size_t b = 0; b < V.geom.bl.size(); ++b) {
      const BlkLev& B = V.geom.bl[b];
      const BlkLev& c = cbl[a.cbl + b];
      for (int z = 0; z <= B.nz + 1; ++z)
        for (int y = 0; y <= B.ny + 1; ++y)
          for (int x = 0; x <= B.nx + 1; ++x) {
            const unsigned long long e = tail_cell(c.off + (long long)z * c.sxy + (long long)y * c.sx + x, x, y, z,
                                                   (int)b);
            const bool gh = x == 0 || y == 0 || z == 0 || x == B.nx + 1 || y == B.ny + 1 || z == B.nz + 1;
            if (gh) ghost.push_back(e);
            else if ((x + y + z) & 1) red.push_back(e);
            else black.push_back(e);
          }
    }
    a.cells = cells.size();
    a.nred = (int)red.size();
    a.nint = (int)(red.size() + black.size());
    cells.insert(cells.end(), red.begin(), red.end());
    cells.insert(cells.end(), black.begin(), black.end());
    a.ghosts = cells.size();
    a.nghost = (int)ghost.size();
    cells.insert(cells.end(), ghost.begin(), ghost.end());
    a.npad = (int)pb;
    // the sweep fill table in compact indices
    std::vector<uint32_t> d, sidx;
    std::string err;
    int rc = build_halo_table(h->blocks, q, kHaloSweep, true, d, sidx, &err);
    if (rc != H3D_OK) return fail(h, rc, err);
    auto compact = [&](uint32_t gi, long long* out) -> bool {
      for (size_t b = 0; b < V.geom.bl.size(); ++b) {
        const BlkLev& B = V.geom.bl[b];
        const long long lo = B.off, hi = B.off + B.sxy * (B.nz + 2);
        if ((long long)gi < lo || (long long)gi >= hi) continue;
        const long long l = (long long)gi - lo;
        const int z = (int)(l / B.sxy), y = (int)((l % B.sxy) / B.sx), x = (int)(l % B.sx);
        if (x > B.nx + 1) return false;
        const BlkLev& c = cbl[a.cbl + b];
        *out = c.off + (long long)z * c.sxy + (long long)y * c.sx + x;
        return true;
      }
      return false;
    };
    a.fdst = fills.size();
    for (uint32_t v : d) {
      long long ci;
      if (!compact(v, &ci)) return H3D_OK;
      fills.push_back((uint32_t)ci);
    }
    a.fsrc = fills.size();
    for (uint32_t v : sidx) {
      long long ci;
      if ((v & kOldFlag) || !compact(v & kIdxMask, &ci)) return H3D_OK;
      fills.push_back((uint32_t)ci);
    }
    a.nfill = (int)d.size();
    at.push_back(a);
  }
  int rc;
  BlkLev* d_cbl = nullptr;
  uint32_t* d_fills = nullptr;
  if ((rc = dalloc(h, &h->d_tail_cells, cells.size())) != H3D_OK || (rc = dalloc(h, &d_cbl, cbl.size())) != H3D_OK ||
      (rc = dalloc(h, &d_fills, std::max<size_t>(fills.size(), 1))) != H3D_OK)
    return rc;
  h->d_tail_cbl = d_cbl;
  h->d_tail_fills = d_fills;
  if (cudaMemcpy(h->d_tail_cells, cells.data(), cells.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(d_cbl, cbl.data(), cbl.size() * sizeof(BlkLev), cudaMemcpyHostToDevice) != cudaSuccess ||
      (!fills.empty() &&
       cudaMemcpy(d_fills, fills.data(), fills.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess))
    return fail(h, H3D_ERR_CUDA, "coarse tail tables");
  std::vector<TailLevel> lv;
  for (int q = g0; q <= Lv; ++q) {
    const Level& V = h->lev[q];
    const At& a = at[q - g0];
    const int k = q - g0;
    TailLevel t{};
    t.gbl = V.d_bl;
    t.cbl = d_cbl + a.cbl;
    t.cells = h->d_tail_cells + a.cells;
    t.ghosts = h->d_tail_cells + a.ghosts;
    t.fdst = d_fills + a.fdst;
    t.fsrc = d_fills + a.fsrc;
    t.nb = (int)V.geom.bl.size();
    t.nint = a.nint;
    t.nred = a.nred;
    t.nghost = a.nghost;
    t.npad = a.npad;
    t.nfill = a.nfill;
    t.phi32[0] = V.phi32[0];
    t.phi32[1] = V.phi32[1];
    t.rhs32 = V.rhs32;
    t.phi64[0] = V.phi64[0];
    t.phi64[1] = V.phi64[1];
    t.rhs64 = V.rhs64;
    t.om = f32_level(h, q) ? h->omega : 1.f;
    t.rb_global = f32_level(h, q) && h->rb_global ? 1 : 0;
    t.s_phi32 = plan.s_phi32[k];
    t.s_rhs32 = plan.s_rhs32[k];
    t.s_phi64 = plan.s_phi64[k];
    t.s_rhs64 = plan.s_rhs64[k];
    lv.push_back(t);
  }
  if ((rc = dalloc(h, &h->d_tail_lv, lv.size())) != H3D_OK) return rc;
  if ((rc = dalloc(h, &h->d_tail_ops, ops.size())) != H3D_OK) return rc;
  if (cudaMemcpy(h->d_tail_lv, lv.data(), lv.size() * sizeof(TailLevel), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_tail_ops, ops.data(), ops.size() * sizeof(TailOp), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(h, H3D_ERR_CUDA, "coarse tail program");
  h->tail_nops = (int)ops.size();
  h->tail_smem = plan.bytes;
  h->tail_zero32.assign(z32.begin() + g0, z32.begin() + Lv + 1);
  h->tail_zero64.assign(z64.begin() + g0, z64.begin() + Lv + 1);
  h->tail_g = g0;
  return H3D_OK;
}

// The fused coarse tail as one cluster of CTAs, CTA b holding block b of
// every tail level: the deepest run of levels g..L (g >= 2, at least two
// levels) whose blocks are all the same size at each level and whose arrays,
// one block of each level, fit one CTA's shared arena; nb <= 16 blocks;
// constant coefficients; sweep fills that read interior cells only.
// coarse_direct: the coarsest level's operator on its interior cells (the
// sweep fill's ghost sources substituted; block-major, x-fastest numbering),
// checked symmetric, and its pseudo-inverse P = (A + sum_c a/n_c 1_c 1_c^T)^-1
// (I - sum_c 1_c 1_c^T / n_c) over the connected components c (the constant
// null vectors of the all-Neumann or periodic operator).  Sets h->d_dense;
// leaves it null when the level does not qualify.
int build_dense_coarse(h3d_mg* h) {
  const int Lv = h->L;
  if (!h->desc.coarse_direct || h->var || h->lmr || h->desc.coarse_sweeps <= 0 || Lv < 2 || f32_level(h, Lv))
    return H3D_OK;
  const LevelGeom G = make_level_geom(h->blocks, Lv, false);
  const int n = (int)G.n_interior;
  // a CTA multiplies n x (n / nb) entries where the sweeps relax n / nb cells
  // coarse_sweeps times: the product pays off below n = 8 coarse_sweeps
  // (measured: 128 and 216 cells faster, 512 cells in one block slower)
  if (n < 1 || n > kDenseMaxCells || n > 8 * h->desc.coarse_sweeps) return H3D_OK;
  std::vector<uint32_t> d, sidx;
  std::string err;
  if (build_halo_table(h->blocks, Lv, kHaloSweep, false, d, sidx, &err) != H3D_OK) return H3D_OK;
  std::vector<uint32_t> src((size_t)G.n_elems, 0xffffffffu);
  for (size_t e = 0; e < d.size(); ++e) src[d[e]] = sidx[e];
  std::vector<int> base(G.bl.size() + 1, 0);
  for (size_t b = 0; b < G.bl.size(); ++b) base[b + 1] = base[b] + G.bl[b].nx * G.bl[b].ny * G.bl[b].nz;
  auto dense_of = [&](uint32_t q) -> int {  // interior cell q -> its dense index (-1: a ghost)
    for (size_t b = 0; b < G.bl.size(); ++b) {
      const BlkLev& B = G.bl[b];
      if ((long long)q < B.off || (long long)q >= B.off + B.sxy * (B.nz + 2)) continue;
      const long long l = (long long)q - B.off;
      const int z = (int)(l / B.sxy), y = (int)((l % B.sxy) / B.sx), x = (int)(l % B.sx);
      if (x < 1 || x > B.nx || y < 1 || y > B.ny || z < 1 || z > B.nz) return -1;
      return base[b] + ((z - 1) * B.ny + (y - 1)) * B.nx + (x - 1);
    }
    return -1;
  };
  std::vector<double> A((size_t)n * n, 0.0);
  for (size_t b = 0; b < G.bl.size(); ++b) {
    const BlkLev& B = G.bl[b];
    for (int z = 1; z <= B.nz; ++z)
      for (int y = 1; y <= B.ny; ++y)
        for (int x = 1; x <= B.nx; ++x) {
          const int i = base[b] + ((z - 1) * B.ny + (y - 1)) * B.nx + (x - 1);
          const int ph = B.phys;
          const double aw = (x == 1 && (ph & 1)) ? 0.0 : B.ax, ae = (x == B.nx && (ph & 2)) ? 0.0 : B.ax;
          const double as = (y == 1 && (ph & 4)) ? 0.0 : B.ay, an = (y == B.ny && (ph & 8)) ? 0.0 : B.ay;
          const double ab = (z == 1 && (ph & 16)) ? 0.0 : B.az, at = (z == B.nz && (ph & 32)) ? 0.0 : B.az;
          A[(size_t)i * n + i] += -(aw + ae + as + an + ab + at);
          const int nbx[6] = {x - 1, x + 1, x, x, x, x}, nby[6] = {y, y, y - 1, y + 1, y, y},
                    nbz[6] = {z, z, z, z, z - 1, z + 1};
          const double c[6] = {aw, ae, as, an, ab, at};
          for (int f = 0; f < 6; ++f) {
            if (c[f] == 0.0) continue;
            uint32_t q = (uint32_t)(B.off + (long long)nbz[f] * B.sxy + (long long)nby[f] * B.sx + nbx[f]);
            int j = dense_of(q);
            if (j < 0) {  // a ghost: its fill source must be an interior cell
              const uint32_t s2 = src[q];
              if (s2 == 0xffffffffu || (s2 & kOldFlag)) return H3D_OK;
              j = dense_of(s2);
              if (j < 0) return H3D_OK;
            }
            A[(size_t)i * n + j] += c[f];
          }
        }
  }
  double amax = 0.0, asym = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      amax = std::max(amax, std::fabs(A[(size_t)i * n + j]));
      asym = std::max(asym, std::fabs(A[(size_t)i * n + j] - A[(size_t)j * n + i]));
    }
  if (!(asym <= 1e-12 * amax) || amax == 0.0) return H3D_OK;
  // connected components of the cell graph
  std::vector<int> comp(n);
  for (int i = 0; i < n; ++i) comp[i] = i;
  std::function<int(int)> root = [&](int i) { return comp[i] == i ? i : (comp[i] = root(comp[i])); };
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (A[(size_t)i * n + j] != 0.0) comp[root(i)] = root(j);
  std::vector<int> csize(n, 0);
  for (int i = 0; i < n; ++i) ++csize[root(i)];
  std::vector<double> R(A);  // A + sum_c amax/n_c 1_c 1_c^T
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (root(i) == root(j)) R[(size_t)i * n + j] += amax / csize[root(i)];
  // Gauss-Jordan inverse with partial pivoting
  std::vector<double> Inv((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Inv[(size_t)i * n + i] = 1.0;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(R[(size_t)i * n + k]) > std::fabs(R[(size_t)piv * n + k])) piv = i;
    if (std::fabs(R[(size_t)piv * n + k]) < 1e-14 * amax) return H3D_OK;
    if (piv != k)
      for (int j = 0; j < n; ++j) {
        std::swap(R[(size_t)k * n + j], R[(size_t)piv * n + j]);
        std::swap(Inv[(size_t)k * n + j], Inv[(size_t)piv * n + j]);
      }
    const double dinv = 1.0 / R[(size_t)k * n + k];
    for (int j = 0; j < n; ++j) {
      R[(size_t)k * n + j] *= dinv;
      Inv[(size_t)k * n + j] *= dinv;
    }
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const double f = R[(size_t)i * n + k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        R[(size_t)i * n + j] -= f * R[(size_t)k * n + j];
        Inv[(size_t)i * n + j] -= f * Inv[(size_t)k * n + j];
      }
    }
  }
  // P = Inv (I - Pi): column j minus the mean of the columns of j's component
  std::vector<double> P((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    std::vector<double> csum(n, 0.0);
    for (int j = 0; j < n; ++j) csum[root(j)] += Inv[(size_t)i * n + j];
    for (int j = 0; j < n; ++j) P[(size_t)i * n + j] = Inv[(size_t)i * n + j] - csum[root(j)] / csize[root(j)];
  }
  TRY(dalloc(h, &h->d_dense, P.size()));
  CU(cudaMemcpy(h->d_dense, P.data(), P.size() * 8, cudaMemcpyHostToDevice));
  h->dense_n = n;
  return H3D_OK;
}

int build_cluster_tail(h3d_mg* h) {
  const int Lv = h->L;
  const int nb = (int)h->blocks.size();
  // (the fused tails restrict and correct between levels of equal-resolution
  // blocks only: none with local mesh refinement)
  if (h->var || h->lmr || nb > kClusterTailMaxBlocks || h->desc.mg_itrsch != 3) return H3D_OK;
  auto al = [](int v) { return (v + 15) & ~15; };
  struct Lay { int npad, nint, s_phi32, s_rhs32, s_phi64, s_rhs64, s_cells, s_fill; };
  std::vector<Lay> lay;
  int g0 = Lv + 1, bytes = 0, scratch_at = 0;
  for (int g = Lv; g >= 2; --g) {
    const Level& V = h->lev[g];
    const BlkLev& B0 = V.geom.bl[0];
    bool same = true;
    for (const auto& B : V.geom.bl) same = same && B.nx == B0.nx && B.ny == B0.ny && B.nz == B0.nz;
    if (!same || B0.nx + 1 > 255 || B0.ny + 1 > 255 || B0.nz + 1 > 255) break;
    // arena with levels g..L (one block each) plus the ghost scratch of the fine levels
    std::vector<Lay> L2;
    int at = 0, scratch = 0;
    for (int q = g; q <= Lv; ++q) {
      const BlkLev& Bq = h->lev[q].geom.bl[0];
      Lay l{};
      l.npad = (Bq.nx + 2) * (Bq.ny + 2) * (Bq.nz + 2);
      l.nint = Bq.nx * Bq.ny * Bq.nz;
      const bool f32 = f32_level(h, q), f64 = !f32 || (h->mixed && q == Lv);
      l.s_phi32 = l.s_rhs32 = l.s_phi64 = l.s_rhs64 = -1;
      if (h->mixed) { l.s_phi32 = at; at = al(at + l.npad * 4); l.s_rhs32 = at; at = al(at + l.nint * 4); }
      if (f64) { l.s_phi64 = at; at = al(at + l.npad * 8); l.s_rhs64 = at; at = al(at + l.nint * 8); }
      if (q < Lv) scratch = std::max(scratch, (l.npad - l.nint) * (f32 ? 4 : 8));
      L2.push_back(l);
    }
    // staged tables: cell + ghost entries of every level, the largest per-block fill list
    int tab = al(at + scratch);
    for (int q = g; q <= Lv; ++q) {
      const BlkLev& Bq = h->lev[q].geom.bl[0];
      const int npad = (Bq.nx + 2) * (Bq.ny + 2) * (Bq.nz + 2);
      L2[q - g].s_cells = tab;
      tab = al(tab + npad * 8);
      L2[q - g].s_fill = tab;
      tab = al(tab + (npad - Bq.nx * Bq.ny * Bq.nz) * 8);  // (dst, src) pairs: a ghost is filled once at most
    }
    const int need = tab + 128;
    if (need > kTailSmemBytes) break;
    g0 = g;
    lay = L2;
    bytes = need;
    scratch_at = at;
  }
  if (g0 > Lv - 1 || Lv - g0 + 1 > kTailMaxLevels) return H3D_OK;
  if (coarse_cluster_fits(nb, bytes) < 1) return H3D_OK;
  std::vector<TailOp> ops;
  std::vector<char> z32, z64;
  TRY(build_dense_coarse(h));
  emit_tail_ops(h, g0, scratch_at, ops, z32, z64, h->d_dense != nullptr);
  // per level: cell tables (block field 0) and per-block fill tables
  std::vector<unsigned long long> cells;
  std::vector<uint32_t> fills;
  std::vector<int> starts;
  struct At { size_t cells, ghosts, fdst, fsrc, fstart; int nred, nint, nghost; };
  std::vector<At> at;
  for (int q = g0; q <= Lv; ++q) {
    const Level& V = h->lev[q];
    const BlkLev& B = V.geom.bl[0];
    const int sx = B.nx + 2, sxy = (B.nx + 2) * (B.ny + 2);
    At a{};
    std::vector<unsigned long long> red, black, ghost;
    for (int z = 0; z <= B.nz + 1; ++z)
      for (int y = 0; y <= B.ny + 1; ++y)
        for (int x = 0; x <= B.nx + 1; ++x) {
          const unsigned long long e = tail_cell((long long)z * sxy + (long long)y * sx + x, x, y, z, 0);
          const bool gh = x == 0 || y == 0 || z == 0 || x == B.nx + 1 || y == B.ny + 1 || z == B.nz + 1;
          if (gh) ghost.push_back(e);
          else if ((x + y + z) & 1) red.push_back(e);
          else black.push_back(e);
        }
    a.cells = cells.size();
    a.nred = (int)red.size();
    a.nint = (int)(red.size() + black.size());
    cells.insert(cells.end(), red.begin(), red.end());
    cells.insert(cells.end(), black.begin(), black.end());
    a.ghosts = cells.size();
    a.nghost = (int)ghost.size();
    cells.insert(cells.end(), ghost.begin(), ghost.end());
    std::vector<uint32_t> d, sidx;
    std::string err;
    int rc = build_halo_table(h->blocks, q, kHaloSweep, true, d, sidx, &err);
    if (rc != H3D_OK) return fail(h, rc, err);
    auto locate = [&](uint32_t gi, int* blk, uint32_t* ci) -> bool {
      for (size_t b = 0; b < V.geom.bl.size(); ++b) {
        const BlkLev& G = V.geom.bl[b];
        const long long lo = G.off, hi = G.off + G.sxy * (G.nz + 2);
        if ((long long)gi < lo || (long long)gi >= hi) continue;
        const long long l = (long long)gi - lo;
        const int z = (int)(l / G.sxy), y = (int)((l % G.sxy) / G.sx), x = (int)(l % G.sx);
        if (x > G.nx + 1) return false;
        *blk = (int)b;
        *ci = (uint32_t)(z * sxy + y * sx + x);
        return true;
      }
      return false;
    };
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> per(nb);
    for (size_t e = 0; e < d.size(); ++e) {
      int bd, bs;
      uint32_t cd, cs;
      if ((sidx[e] & kOldFlag) || !locate(d[e], &bd, &cd) || !locate(sidx[e] & kIdxMask, &bs, &cs)) return H3D_OK;
      per[bd].push_back({cd, ((uint32_t)bs << 24) | cs});
    }
    a.fstart = starts.size();
    a.fdst = fills.size();
    std::vector<uint32_t> fd, fs;
    int acc = 0;
    for (int b = 0; b < nb; ++b) {
      starts.push_back(acc);
      for (auto& pr : per[b]) { fd.push_back(pr.first); fs.push_back(pr.second); }
      acc += (int)per[b].size();
    }
    starts.push_back(acc);
    fills.insert(fills.end(), fd.begin(), fd.end());
    a.fsrc = fills.size();
    fills.insert(fills.end(), fs.begin(), fs.end());
    at.push_back(a);
  }
  int rc;
  uint32_t* d_fills = nullptr;
  int* d_starts = nullptr;
  if ((rc = dalloc(h, &h->d_tail_cells, cells.size())) != H3D_OK ||
      (rc = dalloc(h, &d_fills, std::max<size_t>(fills.size(), 1))) != H3D_OK ||
      (rc = dalloc(h, &d_starts, starts.size())) != H3D_OK)
    return rc;
  h->d_tail_fills = d_fills;
  h->d_tail_starts = d_starts;
  if (cudaMemcpy(h->d_tail_cells, cells.data(), cells.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      (!fills.empty() && cudaMemcpy(d_fills, fills.data(), fills.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(d_starts, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(h, H3D_ERR_CUDA, "cluster tail tables");
  std::vector<TailLevel> lv;
  for (int q = g0; q <= Lv; ++q) {
    const Level& V = h->lev[q];
    const At& a = at[q - g0];
    const Lay& l = lay[q - g0];
    TailLevel t{};
    t.gbl = V.d_bl;
    t.cbl = nullptr;
    t.cells = h->d_tail_cells + a.cells;
    t.ghosts = h->d_tail_cells + a.ghosts;
    t.fdst = d_fills + a.fdst;
    t.fsrc = d_fills + a.fsrc;
    t.fstart = d_starts + a.fstart;
    t.nb = nb;
    t.nint = a.nint;
    t.nred = a.nred;
    t.nghost = a.nghost;
    t.npad = l.npad;
    t.nfill = 0;
    t.phi32[0] = V.phi32[0];
    t.phi32[1] = V.phi32[1];
    t.rhs32 = V.rhs32;
    t.phi64[0] = V.phi64[0];
    t.phi64[1] = V.phi64[1];
    t.rhs64 = V.rhs64;
    t.s_phi32 = l.s_phi32;
    t.s_rhs32 = l.s_rhs32;
    t.s_phi64 = l.s_phi64;
    t.s_rhs64 = l.s_rhs64;
    t.s_cells = l.s_cells;
    t.s_fill = l.s_fill;
    t.dense = q == Lv ? h->d_dense : nullptr;
    t.dense_n = q == Lv ? h->dense_n : 0;
    t.om = f32_level(h, q) ? h->omega : 1.f;
    t.rb_global = f32_level(h, q) && h->rb_global ? 1 : 0;
    lv.push_back(t);
  }
  // every block's fill list must fit its staged region
  for (int q = g0; q <= Lv; ++q) {
    const Lay& l = lay[q - g0];
    const int cap = l.npad - l.nint;
    const size_t f0 = at[q - g0].fstart;
    for (int b = 0; b < nb; ++b)
      if (starts[f0 + b + 1] - starts[f0 + b] > cap) return H3D_OK;
  }
  if ((int)ops.size() > kClusterTailMaxOps) return H3D_OK;
  if ((rc = dalloc(h, &h->d_tail_lv, lv.size())) != H3D_OK) return rc;
  if ((rc = dalloc(h, &h->d_tail_ops, ops.size())) != H3D_OK) return rc;
  if (cudaMemcpy(h->d_tail_lv, lv.data(), lv.size() * sizeof(TailLevel), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_tail_ops, ops.data(), ops.size() * sizeof(TailOp), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(h, H3D_ERR_CUDA, "cluster tail program");
  h->tail_nlev = Lv - g0 + 1;
  h->tail_nops = (int)ops.size();
  h->tail_smem = bytes;
  h->tail_zero32.assign(z32.begin() + g0, z32.begin() + Lv + 1);
  h->tail_zero64.assign(z64.begin() + g0, z64.begin() + Lv + 1);
  h->tail_g = g0;
  h->tail_cluster = nb;
  return H3D_OK;
}

int h3d_mg_destroy(h3d_mg* h) {
  if (!h) return H3D_OK;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  for (auto& kv : h->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto e : kv.second.events) cudaEventDestroy(e);
  }
  for (auto e : h->ev_eager) cudaEventDestroy(e);
  for (size_t g = 1; g < h->lev.size(); ++g) {
    Level& V = h->lev[g];
    void* ps[] = {V.d_bl, V.d_cta_all, V.d_cta_int, V.d_rows_all, V.d_rows_int, V.d_tiles, V.phi64[0], V.phi64[1], V.rhs64, V.phi32[0],
                  V.phi32[1], V.rhs32, V.fx64, V.fy64, V.fz64, V.fx32, V.fy32, V.fz32, V.dens,
                  V.sweep.d_dst, V.sweep.d_src, V.faces.d_dst, V.faces.d_src, V.exch.d_dst, V.exch.d_src,
                  V.bound.d_dst, V.bound.d_src, V.sweep_push.d_dst, V.sweep_push.d_src, V.live.d_dst, V.live.d_src, V.live_push.d_dst, V.live_push.d_src, V.red.d_dst, V.red.d_src, V.d_red_info, V.d_push, V.d_maps, V.d_rmaps, V.d_rtiles, V.d_ptiles, V.d_qtiles, V.d_dtiles, V.d_cstart, V.d_dstart, V.d_pstart, V.seq64, V.seq32, V.d_ztiles, V.lfill.d_dst, V.lfill.d_src, V.d_lfstart,
                  V.xs.d_nodes, V.xs.d_dst, V.xs.d_src, V.xe.d_nodes, V.xe.d_dst, V.xe.d_src, V.xscratch, V.d_rsame,
                  V.d_psame, V.d_prows};
    for (void* p : ps) dfree(p);
  }
  dfree(h->p64[0]);
  dfree(h->p64[1]);
  dfree(h->b64);
  dfree(h->partials);
  dfree(h->d_res);
  dfree(h->d_resb);
  if (h->h_resb) cudaFreeHost(h->h_resb);
  dfree(h->d_h3);
  dfree(h->d_err);
  dfree(h->d_tail_lv);
  dfree(h->d_tail_ops);
  dfree(h->d_dense);
  dfree(h->d_tail_cells);
  dfree(h->d_tail_cbl);
  dfree(h->d_tail_fills);
  dfree(h->d_tail_starts);
  dfree(h->stage[0]);
  dfree(h->stage[1]);
  for (int c = 0; c < 3; ++c) {
    dfree(h->vel[c]);
    dfree(h->vstar[c]);
  }
  dfree(h->d_vdst);
  dfree(h->d_vsrc);
  for (int q = 0; q < 8; ++q) dfree(h->sip[q]);
  dfree(h->sip_pp);
  if (h->h_res) cudaFreeHost(h->h_res);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return H3D_OK;
}

int h3d_mg_create(h3d_mg** out, const h3d_mg_desc* desc) {
  h3d_mg* h = nullptr;
  if (!out || !desc || !desc->blocks || desc->nblocks <= 0) return fail(nullptr, H3D_ERR_ARG, "null descriptor");
  *out = nullptr;
  const h3d_mg_desc& D = *desc;
  if (D.ngrd_gl < 1 || D.ngrd_gl > kMaxLevels) return fail(nullptr, H3D_ERR_BAD_CONFIG, "ngrd_gl out of range");
  if (D.mg_itrsch < 1 || D.mg_itrsch > 3)
    return fail(nullptr, H3D_ERR_BAD_CONFIG, "mg_itrsch must be 1 (GS-lex), 2 (line TDMA) or 3 (red-black GS)");
  if (D.irestr < 0 || D.iproln < 0 || D.irestr + D.iproln < 1)
    return fail(nullptr, H3D_ERR_BAD_CONFIG, "irestr/iproln must be >= 0 with at least one sweep");
  if (D.precision != H3D_PREC_FP64 && D.precision != H3D_PREC_MIXED)
    return fail(nullptr, H3D_ERR_BAD_CONFIG, "unknown precision");
  if (D.coarse_op < 0 || D.coarse_op > 1) return fail(nullptr, H3D_ERR_BAD_CONFIG, "coarse_op must be 0 or 1");
  // local mesh refinement (localparameters.for:28-59): ngrd_gl = ngrid_input +
  // log2(max rdiv), a block of ratio rdiv has ngrid_input + log2(rdiv) levels
  int maxlog = 0;
  bool lmr = false;
  for (int b = 0; b < D.nblocks; ++b) {
    const int r = D.blocks[b].rdiv;
    int lg = 0;
    while ((1 << lg) < r) ++lg;
    if (r < 1 || (1 << lg) != r) return fail(nullptr, H3D_ERR_BAD_CONFIG, "rdiv must be a power of 2");
    maxlog = std::max(maxlog, lg);
  }
  const int ngrid_input = D.ngrd_gl - maxlog;
  if (ngrid_input < 1) return fail(nullptr, H3D_ERR_BAD_CONFIG, "ngrd_gl smaller than log2(max rdiv) + 1");
  for (int b = 0; b < D.nblocks; ++b) {
    const h3d_block_desc& d = D.blocks[b];
    int lg = 0;
    while ((1 << lg) < d.rdiv) ++lg;
    if (d.ngrid != ngrid_input + lg)
      return fail(nullptr, H3D_ERR_BAD_CONFIG,
                  "every block needs ngrid == ngrd_gl - log2(max rdiv) + log2(rdiv) (ngrd_gl without refinement)");
    if (d.ngrid != D.ngrd_gl) lmr = true;
    int pow2 = 1 << (d.ngrid - 1);
    for (int a = 0; a < 3; ++a)
      if (d.n[a] <= 0 || d.n[a] % pow2 != 0)  // localparameters.for:204-209
        return fail(nullptr, H3D_ERR_BAD_CONFIG, "block size not divisible by 2**(ngrid-1)");
    for (int f = 0; f < 6; ++f) {
      if (d.nb_face[f] >= D.nblocks || d.nb_periodic[f] >= D.nblocks)
        return fail(nullptr, H3D_ERR_BAD_CONFIG, "neighbour id out of range");
    }
    for (int e = 0; e < 12; ++e)
      if (d.nb_edge[e] >= D.nblocks) return fail(nullptr, H3D_ERR_BAD_CONFIG, "neighbour id out of range");
    for (int c = 0; c < 8; ++c)
      if (d.nb_corner[c] >= D.nblocks) return fail(nullptr, H3D_ERR_BAD_CONFIG, "neighbour id out of range");
  }
  {
    std::vector<h3d_block_desc> bl(D.blocks, D.blocks + D.nblocks);
    for (int g = 1; g <= D.ngrd_gl && !lmr; ++g) lmr = level_is_lmr(bl, g);
    for (int b = 0; b < D.nblocks; ++b)
      for (int f = 0; f < 6; ++f) {
        const int t = D.blocks[b].nb_periodic[f];
        if (t >= 0 && D.blocks[t].rdiv != D.blocks[b].rdiv)  // exchbc_mgpp copies equal planes only
          return fail(nullptr, H3D_ERR_BAD_CONFIG, "periodic partners need equal rdiv");
      }
  }
  if (lmr && D.var_coef)
    return fail(nullptr, H3D_ERR_BAD_CONFIG, "local mesh refinement with L_LSM coefficients is not supported");
  if (!(D.omega >= 0.f && D.omega < 2.f))
    return fail(nullptr, H3D_ERR_BAD_CONFIG, "omega must be 0 (Gauss-Seidel) or lie in (0, 2)");
  if (D.rb_order != 0 && D.rb_order != 1) return fail(nullptr, H3D_ERR_BAD_CONFIG, "rb_order must be 0 or 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= D.device || D.device < 0)
    return fail(nullptr, H3D_ERR_NO_DEVICE, "no CUDA device");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, D.device) != cudaSuccess || prop.major != 10)
    return fail(nullptr, H3D_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");

  h = new h3d_mg();
  h->device = D.device;
  h->desc = D;
  h->blocks.assign(D.blocks, D.blocks + D.nblocks);
  h->desc.blocks = nullptr;
  if (h->desc.maxcy <= 0) h->desc.maxcy = 30;  // control.cin default
  if (h->desc.inner_cycles <= 0) h->desc.inner_cycles = 2;
  h->L = D.ngrd_gl;
  {
    const char* dbg = std::getenv("H3D_DEBUG_SYNC");
    h->debug_sync = dbg && dbg[0] == '1';
    if (h->debug_sync) h->desc.use_graph = 0;
  }
  h->mixed = D.precision == H3D_PREC_MIXED;
  h->var = D.var_coef != 0;
  h->lmr = lmr;
  h->omega = D.omega > 0.f ? D.omega : 1.f;  // FP32 levels only
  h->rb_global = D.rb_order == 1;
  int rc = H3D_OK;
  auto bail = [&](int r) {
    g_create_error = h->last_error;
    h3d_mg_destroy(h);
    return r;
  };
  if (cudaSetDevice(h->device) != cudaSuccess) return bail(fail(h, H3D_ERR_NO_DEVICE, "cudaSetDevice failed"));
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(h, H3D_ERR_CUDA, "stream create failed"));
  if (init_kernel_attributes() != cudaSuccess || init_kernel_attributes_2() != cudaSuccess)
    return bail(fail(h, H3D_ERR_CUDA, "kernel attributes"));
  h->lev.resize(h->L + 1);
  for (int g = 1; g <= h->L; ++g) {
    Level& V = h->lev[g];
    V.geom = make_level_geom(h->blocks, g, true);
    if ((rc = dalloc(h, &V.d_bl, V.geom.bl.size())) != H3D_OK) return bail(rc);
    if (cudaMemcpy(V.d_bl, V.geom.bl.data(), V.geom.bl.size() * sizeof(BlkLev), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(h, H3D_ERR_CUDA, "copy level geometry"));
    if ((rc = build_cta_table(h, V.geom, false, &V.d_cta_all, &V.ncta_all)) != H3D_OK) return bail(rc);
    if ((rc = build_cta_table(h, V.geom, true, &V.d_cta_int, &V.ncta_int)) != H3D_OK) return bail(rc);
    if ((rc = build_row_table(h, V.geom, false, &V.d_rows_all, &V.nrows_all)) != H3D_OK) return bail(rc);
    if ((rc = build_row_table(h, V.geom, true, &V.d_rows_int, &V.nrows_int)) != H3D_OK) return bail(rc);
    const size_t n = (size_t)V.geom.n_elems;
    const bool need64 = !f32_level(h, g);
    const bool need32 = h->mixed;
    if (need64) {
      if ((rc = dalloc(h, &V.phi64[0], n)) || (rc = dalloc(h, &V.phi64[1], n)) || (rc = dalloc(h, &V.rhs64, n)))
        return bail(rc);
    }
    if (need32) {
      if ((rc = dalloc(h, &V.phi32[0], n)) || (rc = dalloc(h, &V.phi32[1], n)) || (rc = dalloc(h, &V.rhs32, n)))
        return bail(rc);
    }
    if (D.mg_itrsch == 2) {
      if (need64 && (rc = dalloc(h, &V.seq64, n))) return bail(rc);
      if (need32 && (rc = dalloc(h, &V.seq32, n))) return bail(rc);
    }
    if (h->var) {
      if ((rc = dalloc(h, &V.dens, n)) || (rc = dalloc(h, &V.fx64, n)) || (rc = dalloc(h, &V.fy64, n)) ||
          (rc = dalloc(h, &V.fz64, n)))
        return bail(rc);
      if (h->mixed && ((rc = dalloc(h, &V.fx32, n)) || (rc = dalloc(h, &V.fy32, n)) || (rc = dalloc(h, &V.fz32, n))))
        return bail(rc);
      // density defaults to 1 (set_density overrides)
      std::vector<double> ones(n, 1.0);
      if (cudaMemcpy(V.dens, ones.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(h, H3D_ERR_CUDA, "density init"));
    }
    std::vector<uint32_t> d, s;
    std::string err;
    V.expr = h->lmr && level_is_lmr(h->blocks, g);
    if (V.expr) {  // neighbours of different rdv: the fill has arithmetic
      if ((rc = upload_xfill(h, g, kHaloSweep, V.xs)) != H3D_OK) return bail(rc);
    } else {
      if ((rc = build_halo_table(h->blocks, g, kHaloSweep, true, d, s, &err)) != H3D_OK)
        return bail(fail(h, rc, err));
      if ((rc = upload_halo(h, V.sweep, d, s)) != H3D_OK) return bail(rc);
    }
    if (!V.expr && f32_level(h, g) && (rc = build_live(h, V, d, s)) != H3D_OK) return bail(rc);
    if (!V.expr && f32_level(h, g) && !h->var && (rc = build_push(h, V, d, s)) != H3D_OK) return bail(rc);
    if (h->lmr) {  // blocks past their last level restrict by a copy and correct by an add
      if (g >= 2 && (rc = upload_block_list(h, V.geom, V.geom.clamped, false, &V.d_rsame, &V.nrsame,
                                            &V.rsame_cells)) != H3D_OK)
        return bail(rc);
      if (g < h->L) {
        if ((rc = upload_block_list(h, V.geom, V.geom.same_next, true, &V.d_psame, &V.npsame, &V.psame_cells)) !=
            H3D_OK)
          return bail(rc);
        std::vector<int> start(V.geom.bl.size() + 1, 0);
        for (size_t b = 0; b < V.geom.bl.size(); ++b)
          start[b + 1] = start[b] + (V.geom.same_next[b] ? 0 : (V.geom.bl[b].ny + 2) * (V.geom.bl[b].nz + 2));
        V.nprows = start.back();
        if ((rc = dalloc(h, &V.d_prows, start.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_prows, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "prolongation rows"));
      }
    }
    // small levels relax in one fused launch when their fill reads interior cells only;
    // slightly larger ones can still join the fused coarse tail (which has no
    // level-count clamp: not with local mesh refinement)
    if (!V.expr && g > 1 && V.geom.n_interior <= kTailLevelCells &&
        V.geom.bl.size() <= (size_t)kSmallLevelBlocks) {
      bool old = false;
      for (uint32_t v : s) old = old || (v & kOldFlag);
      if (!old) {
        std::vector<int> cs(1, 0);
        for (const auto& B : V.geom.bl) cs.push_back(cs.back() + B.nx * B.ny * B.nz);
        if ((rc = dalloc(h, &V.d_cstart, cs.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_cstart, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "small-level table"));
        V.tailable = !h->lmr;
        V.small = V.geom.n_interior <= kSmallLevelCells;
      }
    }
    // levels whose fill stays inside every block and whose blocks are small
    // enough for one CTA each relax a whole visit in one launch
    if (!V.expr && g > 1 && !V.small) {
      int64_t maxc = 0;
      std::vector<int> owner(V.geom.bl.size());
      for (const auto& B : V.geom.bl) maxc = std::max<int64_t>(maxc, (int64_t)B.nx * B.ny * B.nz);
      auto block_of = [&](uint32_t idx) {
        for (size_t b = 0; b < V.geom.bl.size(); ++b) {
          const BlkLev& B = V.geom.bl[b];
          if ((long long)idx >= B.off && (long long)idx < B.off + (long long)(B.nz + 2) * B.sxy) return (int)b;
        }
        return -1;
      };
      bool local = maxc <= kBlockLocalCells;
      std::vector<std::vector<std::pair<uint32_t, uint32_t>>> per(V.geom.bl.size());
      for (size_t e = 0; local && e < d.size(); ++e) {
        const int bd = block_of(d[e]), bs = block_of(s[e] & kIdxMask);
        if (bd < 0 || bd != bs || (s[e] & kOldFlag)) local = false;  // in place: interior sources only
        else per[bd].push_back({d[e], s[e]});
      }
      if (local) {
        std::vector<uint32_t> ld, ls;
        std::vector<int> st(1, 0);
        for (const auto& v : per) {
          for (const auto& pr : v) { ld.push_back(pr.first); ls.push_back(pr.second); }
          st.push_back((int)ld.size());
        }
        if ((rc = upload_halo(h, V.lfill, ld, ls)) != H3D_OK) return bail(rc);
        if ((rc = dalloc(h, &V.d_lfstart, st.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_lfstart, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "block-local fill table"));
        V.blocal = true;
      }
    }
    if (g == 1 && !V.expr) {  // (with refinement the pressure halo is the sweep's expression fill)
      if ((rc = build_halo_table(h->blocks, g, kHaloFaces, true, d, s, &err)) != H3D_OK) return bail(fail(h, rc, err));
      if ((rc = upload_halo(h, V.faces, d, s)) != H3D_OK) return bail(rc);
    }
    V.f32 = f32_level(h, g);
    V.var = h->var;
    if (g < h->L) {
      // prolongation tiles: plane pairs (2m, 2m+1) of a block, ghost planes included;
      // level 1 also: row tiles of the tiled defect (kProlongRows rows of one plane)
      std::vector<Tile> qt, pt;
      V.pvec32 = V.pvec64 = true;
      for (size_t b = 0; b < V.geom.bl.size(); ++b) {
        const BlkLev& B = V.geom.bl[b];
        const bool even = B.ny % 2 == 0 && B.nz % 2 == 0;
        if (!V.geom.same_next[b]) {  // (blocks whose coarser level is the same size correct by an add)
          V.pvec32 = V.pvec32 && even && B.nx % 4 == 0;
          V.pvec64 = V.pvec64 && even && B.nx % 2 == 0;
          for (int z = 0; z <= B.nz; z += 2) qt.push_back(Tile{(int)b, 0, 0, z});
        }
        if (g == 1)
          for (int z = 0; z <= B.nz + 1; ++z)
            for (int y0 = 0; y0 <= B.ny + 1; y0 += kProlongRows) pt.push_back(Tile{(int)b, 0, y0, z});
      }
      if ((rc = dalloc(h, &V.d_qtiles, qt.size())) != H3D_OK) return bail(rc);
      if (cudaMemcpy(V.d_qtiles, qt.data(), qt.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(h, H3D_ERR_CUDA, "prolongation tiles"));
      V.nqtiles = (int)qt.size();
      if (!pt.empty()) {
        if ((rc = dalloc(h, &V.d_ptiles, pt.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_ptiles, pt.data(), pt.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "defect tiles"));
        V.nptiles = (int)pt.size();
        if ((rc = upload_tile_starts(h, pt, (int)V.geom.bl.size(), &V.d_pstart)) != H3D_OK) return bail(rc);
      }
    }
    const char* zs_env = std::getenv("H3D_ZERO_STENCIL");
    if (f32_level(h, g) && !h->var && h->desc.mg_itrsch == 3 && !(zs_env && zs_env[0] == '0')) {
      // zero-source FP32 sweep tiles: 256 / (nx/4) rows of a block over a chunk of planes
      // (H3D_ZERO_STENCIL=0: the zero-source mode of the tuned sweep kernel instead)
      bool ok = true;
      int maxnz = 0, nyz = 0;
      for (const auto& B : V.geom.bl) {
        ok = ok && B.nx % 4 == 0 && B.nx <= 1024;
        if (!ok) break;
        maxnz = std::max(maxnz, B.nz);
        nyz += (B.ny + 256 / (B.nx / 4) - 1) / (256 / (B.nx / 4));
      }
      if (ok) {
        // about eight CTAs per SM in all, at least four planes a chunk
        V.zzc = std::max(4, std::min(32, (nyz * maxnz + 148 * 8 - 1) / (148 * 8)));
        std::vector<Tile> zt;
        for (size_t b = 0; b < V.geom.bl.size(); ++b) {
          const BlkLev& B = V.geom.bl[b];
          const int rows = 256 / (B.nx / 4);
          for (int z0 = 1; z0 <= B.nz; z0 += V.zzc)
            for (int y0 = 1; y0 <= B.ny; y0 += rows) zt.push_back(Tile{(int)b, 1, y0, z0});
        }
        if ((rc = dalloc(h, &V.d_ztiles, zt.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_ztiles, zt.data(), zt.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "zero-sweep tiles"));
        V.nztiles = (int)zt.size();
      }
    }
    if (g == 1 && !h->var) {  // z-march defect tiles: 8 rows of a block over a chunk of planes
      int maxnx = 0, maxnz = 0, nyt = 0;
      bool even = true;
      for (const auto& B : V.geom.bl) {
        maxnx = std::max(maxnx, B.nx);
        maxnz = std::max(maxnz, B.nz);
        even = even && B.nx % 2 == 0;
        nyt += (B.ny + defect_march_rows() - 1) / defect_march_rows();
      }
      V.dgp = !even ? 0 : maxnx <= 64 ? 1 : maxnx <= 128 ? 2 : maxnx <= 256 ? 4 : 0;
      if (V.dgp) {
        // about six CTAs per SM in all, chunks of at least four planes
        const int chunks = std::max(1, std::min((148 * 6 + nyt - 1) / nyt, maxnz / 4));
        V.dzc = std::max(1, (maxnz + chunks - 1) / chunks);
        std::vector<Tile> dt;
        for (size_t b = 0; b < V.geom.bl.size(); ++b) {
          const BlkLev& B = V.geom.bl[b];
          for (int z0 = 1; z0 <= B.nz; z0 += V.dzc)
            for (int y0 = 1; y0 <= B.ny; y0 += defect_march_rows()) dt.push_back(Tile{(int)b, 0, y0, z0});
        }
        if ((rc = dalloc(h, &V.d_dtiles, dt.size())) != H3D_OK) return bail(rc);
        if (cudaMemcpy(V.d_dtiles, dt.data(), dt.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess)
          return bail(fail(h, H3D_ERR_CUDA, "defect tiles"));
        V.ndtiles = (int)dt.size();
        if ((rc = upload_tile_starts(h, dt, (int)V.geom.bl.size(), &V.d_dstart)) != H3D_OK) return bail(rc);
      }
    }
    if ((rc = build_tensor_maps(h, g)) != H3D_OK) return bail(rc);
    if (g >= 2 && (rc = build_restrict_tiles(h, V)) != H3D_OK) return bail(rc);
    int var_, zc;
    default_tile(V, &var_, &zc);
    if ((rc = build_tiles(h, V, var_, zc)) != H3D_OK) return bail(rc);
    // bytes of one sweep: read phi + rhs, write phi (+3 face arrays when variable)
    double w = f32_level(h, g) ? 4.0 : 8.0;
    V.sweep_bytes = (double)V.geom.n_interior * w * (3.0 + (h->var ? 3.0 : 0.0));
    V.sweep_bytes_zero = (double)V.geom.n_interior * w * (2.0 + (h->var ? 3.0 : 0.0));
  }
  if ((rc = build_cluster_tail(h)) != H3D_OK) return bail(rc);
  if (!h->tail_g && (rc = build_tail(h)) != H3D_OK) return bail(rc);
  const size_t n1 = (size_t)h->lev[1].geom.n_elems;
  if ((rc = dalloc(h, &h->p64[0], n1)) || (rc = dalloc(h, &h->p64[1], n1)) || (rc = dalloc(h, &h->b64, n1)))
    return bail(rc);
  h->npartials = std::max(std::max(std::max(h->lev[1].ncta_all, h->lev[1].ncta_int), kDefectCtas),
                          std::max(h->lev[1].nptiles, h->lev[1].ndtiles));
  if ((rc = dalloc(h, &h->partials, 4 * (size_t)h->npartials)) || (rc = dalloc(h, &h->d_res, 4))) return bail(rc);
  if ((rc = dalloc(h, &h->d_resb, 4 * h->blocks.size())) != H3D_OK) return bail(rc);
  if (cudaMallocHost((void**)&h->h_resb, 4 * sizeof(double) * h->blocks.size()) != cudaSuccess)
    return bail(fail(h, H3D_ERR_OOM, "pinned per-block result buffer"));
  if (cudaMallocHost((void**)&h->h_res, 4 * sizeof(double)) != cudaSuccess)
    return bail(fail(h, H3D_ERR_OOM, "pinned result buffer"));
  std::vector<double> h3;
  for (const auto& d : h->blocks) { h3.push_back(d.h[0]); h3.push_back(d.h[1]); h3.push_back(d.h[2]); }
  if ((rc = dalloc(h, &h->d_h3, h3.size())) != H3D_OK) return bail(rc);
  if ((rc = dalloc(h, &h->d_err, 1)) != H3D_OK) return bail(rc);
  if (cudaMemcpy(h->d_h3, h3.data(), h3.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(h, H3D_ERR_CUDA, "copy spacings"));
  if (cudaStreamSynchronize(h->st) != cudaSuccess) return bail(fail(h, H3D_ERR_CUDA, "set-up sync"));
  if (!h->var) h->coeffs_ready = true;
  *out = h;
  return H3D_OK;
}

int h3d_mg_set_density(h3d_mg* h, int32_t ib, const double* dens) {
  if (!h || !dens || ib < 0 || ib >= (int)h->blocks.size()) return H3D_ERR_ARG;
  if (!h->var) return fail(h, H3D_ERR_ARG, "handle was created with var_coef = 0");
  TRY(check_block_host_dims(h, h->blocks[ib]));
  CU(cudaSetDevice(h->device));
  TRY(copy_field_3d(h, true, h->lev[1].dens, h->lev[1].geom.bl[ib], const_cast<double*>(dens), h->blocks[ib], true));
  CU(cudaStreamSynchronize(h->st));
  h->coeffs_ready = false;
  return H3D_OK;
}

int h3d_mg_coeff(h3d_mg* h) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  if (h->var) {
    for (int g = 1; g <= h->L; ++g) {
      Level& V = h->lev[g];
      CellTab ca{V.d_cta_all, (int)V.geom.bl.size(), V.ncta_all};
      if (g > 1) {
        Level& F = h->lev[g - 1];
        CellTab ct{V.d_cta_int, (int)V.geom.bl.size(), V.ncta_int};
        CU(launch_dens_restrict(F.d_bl, V.d_bl, ct, F.dens, V.dens, h->st));
        if (h->desc.coarse_op == 1)
          CU(launch_face_coef_sum(F.d_bl, V.d_bl, ca, F.fx64, F.fy64, F.fz64, V.fx64, V.fy64, V.fz64, h->st));
      }
      if (g == 1 || h->desc.coarse_op == 0)
        CU(launch_face_coef(V.d_bl, ca, V.dens, h->d_h3, V.fx64, V.fy64, V.fz64, h->st));
      if (h->mixed) {
        CU(launch_convert_d2f(V.fx64, V.fx32, V.geom.n_elems, h->st));
        CU(launch_convert_d2f(V.fy64, V.fy32, V.geom.n_elems, h->st));
        CU(launch_convert_d2f(V.fz64, V.fz32, V.geom.n_elems, h->st));
      }
    }
    CU(cudaStreamSynchronize(h->st));
  }
  // autotune the smoother tiles of the large levels once coefficients exist
  if (h->desc.mg_itrsch == 3)  // the tuned variants are red-black sweeps
    for (int g = 1; g <= h->L; ++g) TRY(autotune_level(h, g));
  for (int g = 2; g <= h->L; ++g) TRY(autotune_restrict(h, g));
  CU(cudaStreamSynchronize(h->st));
  h->coeffs_ready = true;
  return H3D_OK;
}

static int ensure_velocity(h3d_mg* h);
static int ensure_sip(h3d_mg* h);
static double* velocity_field(h3d_mg* h, int field);

static int ensure_coeffs(h3d_mg* h) {
  if (!h->coeffs_ready) return h3d_mg_coeff(h);
  return H3D_OK;
}

int h3d_mg_upload(h3d_mg* h, int32_t field, int32_t ib, const double* host) {
  if (!h || !host || ib < 0 || ib >= (int)h->blocks.size()) return H3D_ERR_ARG;
  TRY(check_block_host_dims(h, h->blocks[ib]));
  CU(cudaSetDevice(h->device));
  const BlkLev& B = h->lev[1].geom.bl[ib];
  if (field == H3D_FIELD_P) TRY(copy_field_3d(h, true, h->p64[h->pc], B, const_cast<double*>(host), h->blocks[ib], true));
  else if (field == H3D_FIELD_B) TRY(copy_field_3d(h, true, h->b64, B, const_cast<double*>(host), h->blocks[ib], false));
  else if (field >= H3D_FIELD_U && field <= H3D_FIELD_WSTAR) {
    TRY(ensure_velocity(h));
    TRY(copy_field_3d(h, true, velocity_field(h, field), B, const_cast<double*>(host), h->blocks[ib], true));
  } else if (field == H3D_FIELD_PP) {
    TRY(ensure_sip(h));
    TRY(copy_field_3d(h, true, h->sip_pp, B, const_cast<double*>(host), h->blocks[ib], true));
  } else
    return H3D_ERR_ARG;
  return H3D_OK;
}

int h3d_mg_download(h3d_mg* h, int32_t field, int32_t ib, double* host) {
  if (!h || !host || ib < 0 || ib >= (int)h->blocks.size()) return H3D_ERR_ARG;
  TRY(check_block_host_dims(h, h->blocks[ib]));
  CU(cudaSetDevice(h->device));
  const BlkLev& B = h->lev[1].geom.bl[ib];
  if (field == H3D_FIELD_P) TRY(copy_field_3d(h, false, h->p64[h->pc], B, host, h->blocks[ib], true));
  else if (field == H3D_FIELD_B) TRY(copy_field_3d(h, false, h->b64, B, host, h->blocks[ib], false));
  else if (field >= H3D_FIELD_U && field <= H3D_FIELD_WSTAR) {
    TRY(ensure_velocity(h));
    TRY(copy_field_3d(h, false, velocity_field(h, field), B, host, h->blocks[ib], true));
  } else if (field == H3D_FIELD_PP) {
    TRY(ensure_sip(h));
    TRY(copy_field_3d(h, false, h->sip_pp, B, host, h->blocks[ib], true));
  } else
    return H3D_ERR_ARG;
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_zero_field(h3d_mg* h, int32_t field) {
  if (!h || (field != H3D_FIELD_P && field != H3D_FIELD_B)) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  double* a = field == H3D_FIELD_P ? h->p64[h->pc] : h->b64;
  CU(cudaMemsetAsync(a, 0, (size_t)h->lev[1].geom.n_elems * sizeof(double), h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_residual(h3d_mg* h, double* rr, double* bb, double* rinf) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  TRY(pressure_halo(h));
  Exec ex{h};
  double save = h->mean_b;
  h->mean_b = 0.0;
  int rc = ex.defect(false);
  h->mean_b = save;
  TRY(rc);
  CU(cudaStreamSynchronize(h->st));
  if (rr) *rr = h->h_res[0];
  if (bb) *bb = h->h_res[1];
  if (rinf) *rinf = h->h_res[2];
  return H3D_OK;
}

int h3d_mg_solve_resident(h3d_mg* h, const h3d_solve_opts* opts, h3d_solve_info* info) {
  if (!h || !opts) return H3D_ERR_ARG;
  if (opts->stop_rule < 0 || opts->stop_rule > 2) return fail(h, H3D_ERR_ARG, "stop_rule must be 0, 1 or 2");
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  const int nb = (int)h->blocks.size();
  struct PerBlock {  // restores the handle's defect mode on every exit
    h3d_mg* h;
    ~PerBlock() { h->per_block = false; }
  } pb_guard{h};
  h->per_block = opts->stop_rule == 2 && nb > 1;
  h3d_solve_info I{};
  const int maxcy = opts->maxcy > 0 ? opts->maxcy : h->desc.maxcy;
  const int inner = h->mixed ? h->desc.inner_cycles : 1;
  h->history.clear();
  cudaEvent_t t0, t1;
  CU(cudaEventCreate(&t0));
  CU(cudaEventCreate(&t1));
  int64_t k0 = h->kernels;
  CU(cudaEventRecord(t0, h->st));
  Level& V = h->lev[1];
  // pressure halo (exchange(4) + pbound, newsolv_mg.for:51-52)
  TRY(pressure_halo(h));
  h->kernels += 1;
  Exec ex{h};
  TRY(ex.chk("pressure halo", 1));
  h->mean_b = 0.0;
  if (h->mixed && is_all_neumann(h) && !h->lmr) {  // (with refinement the operator's left null vector is not constant)
    // FP64 null-space handling: the compatible part of b has zero mean; the
    // FP32 cycles see the defect with the mean of b removed.
    RowTab rt{V.d_rows_int, (int)V.geom.bl.size(), V.nrows_int};
    int np = 0;
    CU(launch_sum_interior(V.d_bl, rt, h->b64, h->partials, &np, h->st));
    TRY(ex.chk("sum b", 1));
    CU(launch_reduce4(h->partials, np, h->d_res, h->st));
    TRY(ex.chk("reduce sum b", 1));
    CU(cudaMemcpyAsync(h->h_res, h->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CU(cudaStreamSynchronize(h->st));
    h->mean_b = h->h_res[0] / (double)V.geom.n_interior;
    h->kernels += 2;
  }
  TRY(ex.defect(false));
  CU(cudaStreamSynchronize(h->st));
  double bb = h->h_res[1];
  I.bnorm = std::sqrt(bb);
  const double bn = I.bnorm > 0 ? I.bnorm : 1.0;
  double rel = std::sqrt(h->h_res[0]) / bn, rinf = h->h_res[2];
  // per-block relative residuals (stop_rule 2): ||r_b|| / ||b_b|| of every block
  std::vector<double> bnb(nb, bn);
  if (h->per_block)
    for (int b = 0; b < nb; ++b) bnb[b] = h->h_resb[4 * b + 1] > 0 ? std::sqrt(h->h_resb[4 * b + 1]) : 1.0;
  auto block_max = [&]() {
    if (!h->per_block) return rel;
    double m = 0;
    for (int b = 0; b < nb; ++b) {
      const double v = std::sqrt(h->h_resb[4 * b]) / bnb[b];
      if (!(v <= m)) m = v;  // keeps a NaN
    }
    return m;
  };
  double relb = block_max();
  if (opts->record_history) h->history.push_back(opts->stop_rule == 2 ? relb : rel);
  int status = 1, iter = 0;
  if (opts->stop_rule == 0 && rel <= opts->tol) status = 0;
  if (opts->stop_rule == 2 && relb <= opts->tol) status = 0;
  double prof_ms = 0, prof_bytes = 0;
  int64_t prof_n = 0;
  while (status != 0 && iter < maxcy) {
    TRY(run_iteration(h, inner, &prof_ms, &prof_n, &prof_bytes));
    iter += 1;
    I.cycles += inner;
    rel = std::sqrt(h->h_res[0]) / bn;
    rinf = h->h_res[2];
    relb = block_max();
    if (opts->record_history) h->history.push_back(opts->stop_rule == 2 ? relb : rel);
    if (!std::isfinite(rel) || rel > 1e8 || !std::isfinite(relb)) { status = 2; break; }
    if (opts->stop_rule == 0 && rel <= opts->tol) status = 0;
    if (opts->stop_rule == 1 && rinf < opts->tol && iter > 1) status = 0;  // newsolv_mg.for:57
    if (opts->stop_rule == 2 && relb <= opts->tol) status = 0;
  }
  if (opts->remove_mean) {
    RowTab rt{V.d_rows_int, (int)V.geom.bl.size(), V.nrows_int};
    int np = 0;
    CU(launch_sum_interior(V.d_bl, rt, h->p64[h->pc], h->partials, &np, h->st));
    CU(launch_reduce4(h->partials, np, h->d_res, h->st));
    CU(launch_shift(h->p64[h->pc], V.geom.n_elems, h->d_res, 1.0 / (double)V.geom.n_interior, h->st));
    h->kernels += 3;
  }
  CU(cudaEventRecord(t1, h->st));
  CU(cudaEventSynchronize(t1));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  I.outer = iter;
  I.relres = rel;
  I.relres_block_max = relb;
  I.rmax = rinf;
  I.device_ms = ms;
  I.smoother_ms = prof_ms;
  I.smoother_launches = prof_n;
  I.smoother_bytes = prof_bytes;
  I.kernel_launches = h->kernels - k0;
  if (info) *info = I;
  TRY(check_device_error(h));
  if (status == 2) return fail(h, H3D_ERR_DIVERGED, "residual is not finite or grew beyond 1e8");
  if (status != 0) return fail(h, H3D_ERR_NOT_CONVERGED, "not converged within maxcy cycles");
  return H3D_OK;
}

int h3d_mg_newsolv(h3d_mg* h, double* const* p, const double* const* b, const h3d_solve_opts* opts,
                   h3d_solve_info* info) {
  if (!h || !p || !b || !opts) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  for (int ib = 0; ib < (int)h->blocks.size(); ++ib) {
    TRY(stage_in(h, 0, ib, p[ib], h->p64[h->pc], true));
    TRY(stage_in(h, 1, ib, b[ib], h->b64, false));
  }
  int rc = h3d_mg_solve_resident(h, opts, info);
  if (rc != H3D_OK && rc != H3D_ERR_NOT_CONVERGED) return rc;
  for (int ib = 0; ib < (int)h->blocks.size(); ++ib) TRY(stage_out(h, 0, ib, p[ib], h->p64[h->pc], true));
  CU(cudaStreamSynchronize(h->st));
  return rc;
}

int h3d_mg_history(h3d_mg* h, double* out, int32_t cap, int32_t* n) {
  if (!h || !n) return H3D_ERR_ARG;
  int k = (int)std::min<size_t>(h->history.size(), (size_t)std::max(cap, 0));
  if (out)
    for (int q = 0; q < k; ++q) out[q] = h->history[q];
  *n = (int)h->history.size();
  return H3D_OK;
}

// ---------------------------------------------------------- the projection
// Face ghosts of the velocity components after calvel (exchange(1..3) at
// equal resolution: exchange_bc.for then exchange.for:302-1650, ghost layer
// 0 on the interior rows): a low-side ghost takes the source block's last
// interior plane, a high-side ghost its first; the source is the face
// neighbour, else (bc = 5) the block itself when it has no neighbour on
// either side of that axis, else its periodic partner.  Physical walls keep
// their values.  Every entry reads an interior cell, so the order is free.
static int build_vel_table(h3d_mg* h) {
  const LevelGeom& G = h->lev[1].geom;
  std::vector<uint32_t> dst, src;
  const int nb = (int)h->blocks.size();
  for (int b = 0; b < nb; ++b) {
    const h3d_block_desc& d = h->blocks[b];
    const BlkLev& B = G.bl[b];
    for (int f = 0; f < 6; ++f) {
      if (B.phys & (1 << f)) continue;
      int sb = -1;
      if (d.nb_face[f] >= 0) sb = d.nb_face[f];
      else if (d.bc[f] == 5) sb = d.nb_face[f ^ 1] < 0 ? b : d.nb_periodic[f];
      if (sb < 0) continue;
      const BlkLev& S = G.bl[sb];
      const int ax = f / 2, hi = f & 1;
      const int nB[3] = {B.nx, B.ny, B.nz}, nS[3] = {S.nx, S.ny, S.nz};
      for (int a = 0; a < 3; ++a)
        if (a != ax && nB[a] != nS[a]) return fail(h, H3D_ERR_BAD_CONFIG, "velocity exchange: face extents differ");
      const int ta = (ax + 1) % 3, tb = (ax + 2) % 3;
      for (int q = 1; q <= nB[tb]; ++q)
        for (int r = 1; r <= nB[ta]; ++r) {
          int cd[3], cs[3];
          cd[ta] = cs[ta] = r;
          cd[tb] = cs[tb] = q;
          cd[ax] = hi ? nB[ax] + 1 : 0;
          cs[ax] = hi ? 1 : nS[ax];
          dst.push_back((uint32_t)(B.off + (long long)cd[2] * B.sxy + (long long)cd[1] * B.sx + cd[0]));
          src.push_back((uint32_t)(S.off + (long long)cs[2] * S.sxy + (long long)cs[1] * S.sx + cs[0]));
        }
    }
  }
  h->nvfill = (int64_t)dst.size();
  if (h->nvfill == 0) return H3D_OK;
  TRY(dalloc(h, &h->d_vdst, dst.size()));
  TRY(dalloc(h, &h->d_vsrc, src.size()));
  CU(cudaMemcpyAsync(h->d_vdst, dst.data(), dst.size() * 4, cudaMemcpyHostToDevice, h->st));
  CU(cudaMemcpyAsync(h->d_vsrc, src.data(), src.size() * 4, cudaMemcpyHostToDevice, h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

static int ensure_face_table(h3d_mg* h) {
  if (h->d_vdst) return H3D_OK;  // (a layout without block faces rebuilds an empty table)
  return build_vel_table(h);
}

static int ensure_velocity(h3d_mg* h) {
  if (h->lmr)
    return fail(h, H3D_ERR_BAD_CONFIG, "the projection loop with local mesh refinement is not supported");
  if (h->vel[0]) return H3D_OK;
  const size_t n = (size_t)h->lev[1].geom.n_elems;
  for (int c = 0; c < 3; ++c) {
    TRY(dalloc(h, &h->vel[c], n));
    TRY(dalloc(h, &h->vstar[c], n));
  }
  return ensure_face_table(h);
}

static double* velocity_field(h3d_mg* h, int field) {
  if (field >= H3D_FIELD_U && field <= H3D_FIELD_W) return h->vel[field - H3D_FIELD_U];
  if (field >= H3D_FIELD_USTAR && field <= H3D_FIELD_WSTAR) return h->vstar[field - H3D_FIELD_USTAR];
  if (field == H3D_FIELD_PP) return h->sip_pp;
  return nullptr;
}

// ---------------------------------------------------------------- SIP
static int ensure_sip(h3d_mg* h) {
  if (h->var) return fail(h, H3D_ERR_BAD_CONFIG, "SIP: constant coefficients only (press.for:407-438)");
  if (h->lmr) return fail(h, H3D_ERR_BAD_CONFIG, "SIP with local mesh refinement is not supported");
  if ((int)h->blocks.size() > h->npartials) return fail(h, H3D_ERR_BAD_CONFIG, "SIP: too many blocks");
  if (h->sip_pp) return H3D_OK;
  TRY(ensure_face_table(h));
  const size_t n = (size_t)h->lev[1].geom.n_elems;
  for (int q = 0; q < 8; ++q) TRY(dalloc(h, &h->sip[q], n));
  TRY(dalloc(h, &h->sip_pp, n));
  return H3D_OK;
}

// sipsol(44) (sipsol.for:2-205) on the resident correction with the resident
// right-hand side (H3D_FIELD_B): factors, then at most nswp sweeps, each
// followed by exchange(44) (face ghosts; walls untouched) and the stop test
// on sum |res| relative to the first sweep (<= 0.001, or changing by at most
// 0.00001).  *nsweep gets the reference's sweep count.
static int sip_run(h3d_mg* h, int nswp, int* nsweep, double* resab_last) {
  Level& V = h->lev[1];
  const int nb = (int)V.geom.bl.size();
  SipArrays a{h->sip[0], h->sip[1], h->sip[2], h->sip[3], h->sip[4], h->sip[5], h->sip[6], h->sip[7]};
  CU(launch_sip_factor(V.d_bl, nb, a, h->st));
  h->kernels += 1;
  const double small = 1e-20;
  double relast = 0.0, res1 = 0.0, resab = 0.0;
  int ns;
  for (ns = 1; ns <= nswp; ++ns) {
    CU(launch_sip_sweep(V.d_bl, nb, a, h->sip_pp, h->b64, h->partials, h->st));
    CU(launch_gather1(h->d_vdst, h->d_vsrc, h->nvfill, h->sip_pp, h->st));
    CU(launch_reduce4(h->partials, nb, h->d_res, h->st));
    CU(cudaMemcpyAsync(h->h_res, h->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CU(cudaStreamSynchronize(h->st));
    h->kernels += 3;
    resab = h->h_res[0];
    if (!std::isfinite(resab)) return fail(h, H3D_ERR_DIVERGED, "SIP residual is not finite");
    if (ns == 1) res1 = resab;
    const double rsm = resab / (res1 + small);
    const double reldif = std::fabs(rsm - relast);
    relast = rsm;
    if (rsm <= 0.001) break;
    if (reldif <= 0.00001) break;
  }
  if (ns > nswp) ns = nswp;
  if (nsweep) *nsweep = ns;
  if (resab_last) *resab_last = resab;
  return H3D_OK;
}

int h3d_mg_sipsol(h3d_mg* h, int32_t nswp, int32_t* nsweep, double* resab) {
  if (!h || nswp < 1) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_sip(h));
  int ns = 0;
  TRY(sip_run(h, nswp, &ns, resab));
  if (nsweep) *nsweep = ns;
  return H3D_OK;
}

int h3d_mg_pressure_1sweep(h3d_mg* h, double dt, double alfapr, double eps, int32_t niter, int32_t nswp,
                           h3d_solve_info* info) {
  if (!h || niter < 1 || nswp < 1) return H3D_ERR_ARG;
  if (!(dt > 0)) return fail(h, H3D_ERR_ARG, "dt must be positive");
  CU(cudaSetDevice(h->device));
  TRY(ensure_sip(h));
  TRY(ensure_velocity(h));
  Level& V = h->lev[1];
  RowTab ra{V.d_rows_all, (int)V.geom.bl.size(), V.nrows_all};
  h3d_solve_info I{};
  h->history.clear();
  cudaEvent_t t0, t1;
  CU(cudaEventCreate(&t0));
  CU(cudaEventCreate(&t1));
  const int64_t k0 = h->kernels;
  CU(cudaEventRecord(t0, h->st));
  const size_t bytes = (size_t)V.geom.n_elems * sizeof(double);
  CU(cudaMemsetAsync(h->sip_pp, 0, bytes, h->st));  // press.for:402
  TRY(h3d_mg_calvel(h, dt, alfapr));               // :439
  int iter = 0, total = 0;
  double rmax = 0.0, su2 = 0.0;
  for (;;) {  // :441-472
    iter += 1;
    TRY(h3d_mg_calmas(h, dt, &rmax, &su2));
    h->history.push_back(rmax);
    if (!std::isfinite(rmax)) break;
    if (rmax < eps && iter > 1) break;
    int ns = 0;
    TRY(sip_run(h, nswp, &ns, nullptr));
    total += ns;
    double* p = h->p64[h->pc];
    CU(launch_padd<double>(V.d_bl, ra, p, h->sip_pp, h->st));  // p = p + (pp - ppref), ppref = 0
    CU(cudaMemsetAsync(h->sip_pp, 0, bytes, h->st));
    CU(launch_fill<double>(V.faces.d_dst, V.faces.d_src, V.faces.n, p, p, p, false, h->st));  // exchange(4), pbound
    h->kernels += 2;
    TRY(h3d_mg_calvel(h, dt, alfapr));
    if (!(iter < niter)) break;
  }
  CU(cudaEventRecord(t1, h->st));
  CU(cudaEventSynchronize(t1));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  I.outer = iter;
  I.cycles = total;
  I.rmax = rmax;
  I.relres = std::sqrt(su2);
  I.relres_block_max = I.relres;
  I.device_ms = ms;
  I.kernel_launches = h->kernels - k0;
  if (info) *info = I;
  TRY(check_device_error(h));
  if (!std::isfinite(rmax) || rmax > 10.0) return fail(h, H3D_ERR_DIVERGED, "rmax not finite or above 10");
  return H3D_OK;
}

// Cached graphs of projection iterations hold dt*alfapr and dt as kernel
// arguments: drop them when either changes.
static void set_projection_scalars(h3d_mg* h, double dt, double alfapr) {
  const double dtal = dt * alfapr;
  if (dtal == h->proj_dtal && dt == h->proj_dt) return;
  for (auto it = h->graphs.begin(); it != h->graphs.end();) {
    if (it->first[0] & 4) {
      if (it->second.exec) cudaGraphExecDestroy(it->second.exec);
      for (auto e : it->second.events) cudaEventDestroy(e);
      it = h->graphs.erase(it);
    } else {
      ++it;
    }
  }
  h->proj_dtal = dtal;
  h->proj_dt = dt;
}

int h3d_mg_calvel(h3d_mg* h, double dt, double alfapr) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_velocity(h));
  set_projection_scalars(h, dt, alfapr);
  Level& V = h->lev[1];
  RowTab ri{V.d_rows_int, (int)V.geom.bl.size(), V.nrows_int};
  CU(launch_calvel(h->var, V.d_bl, ri, h->d_h3, h->p64[h->pc], V.dens, h->vstar[0], h->vstar[1], h->vstar[2],
                   h->vel[0], h->vel[1], h->vel[2], h->proj_dtal, h->st));
  CU(launch_gather3(h->d_vdst, h->d_vsrc, h->nvfill, h->vel[0], h->vel[1], h->vel[2], h->st));
  CU(cudaStreamSynchronize(h->st));
  return check_device_error(h);
}

int h3d_mg_calmas(h3d_mg* h, double dt, double* rmax, double* su2) {
  if (!h) return H3D_ERR_ARG;
  if (!(dt > 0)) return fail(h, H3D_ERR_ARG, "dt must be positive");
  CU(cudaSetDevice(h->device));
  TRY(ensure_velocity(h));
  Level& V = h->lev[1];
  RowTab ri{V.d_rows_int, (int)V.geom.bl.size(), V.nrows_int};
  int np = 0;
  if (h->mixed)
    CU(launch_calmas<float>(h->var, V.d_bl, ri, h->d_h3, h->vel[0], h->vel[1], h->vel[2], dt, h->b64, V.rhs32,
                            h->partials, &np, h->st));
  else
    CU(launch_calmas<double>(h->var, V.d_bl, ri, h->d_h3, h->vel[0], h->vel[1], h->vel[2], dt, h->b64, V.rhs64,
                             h->partials, &np, h->st));
  CU(launch_reduce4(h->partials, np, h->d_res, h->st));
  CU(cudaMemcpyAsync(h->h_res, h->d_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CU(cudaStreamSynchronize(h->st));
  if (su2) *su2 = h->h_res[0];
  if (rmax) *rmax = h->h_res[2];
  return H3D_OK;
}

int h3d_mg_pbound(h3d_mg* h) {
  if (!h) return H3D_ERR_ARG;
  if (h->lmr) return fail(h, H3D_ERR_BAD_CONFIG, "pbound with local mesh refinement is not supported");
  CU(cudaSetDevice(h->device));
  Level& V = h->lev[1];
  double* p = h->p64[h->pc];
  CU(launch_fill<double>(V.faces.d_dst, V.faces.d_src, V.faces.n, p, p, p, false, h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_project_resident(h3d_mg* h, double dt, double alfapr, const h3d_solve_opts* opts,
                            h3d_solve_info* info) {
  if (!h || !opts) return H3D_ERR_ARG;
  if (opts->stop_rule != 0 && opts->stop_rule != 1)
    return fail(h, H3D_ERR_ARG, "the projection stops on rule 0 or 1");
  if (!(dt > 0)) return fail(h, H3D_ERR_ARG, "dt must be positive");
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  TRY(ensure_velocity(h));
  struct ProjGuard {  // restores the handle's defect mode on every exit
    h3d_mg* h;
    ~ProjGuard() { h->proj = false; }
  } guard{h};
  set_projection_scalars(h, dt, alfapr);
  h->proj = true;
  h->per_block = false;
  h3d_solve_info I{};
  const int maxcy = opts->maxcy > 0 ? opts->maxcy : h->desc.maxcy;
  const int inner = h->mixed ? h->desc.inner_cycles : 1;
  h->history.clear();
  cudaEvent_t t0, t1;
  CU(cudaEventCreate(&t0));
  CU(cudaEventCreate(&t1));
  int64_t k0 = h->kernels;
  CU(cudaEventRecord(t0, h->st));
  Exec ex{h};
  TRY(ex.vel_defect());  // calvel, calmas on the given p (newsolv_mg.for:16-17)
  CU(cudaStreamSynchronize(h->st));
  I.bnorm = std::sqrt(h->h_res[0]);
  const double bn = I.bnorm > 0 ? I.bnorm : 1.0;
  double rel = std::sqrt(h->h_res[0]) / bn, rmax = h->h_res[2];
  if (opts->record_history) h->history.push_back(opts->stop_rule == 1 ? rmax : rel);
  int status = 1, iter = 0;
  if (opts->stop_rule == 0 && rel <= opts->tol) status = 0;
  double prof_ms = 0, prof_bytes = 0;
  int64_t prof_n = 0;
  while (status != 0 && iter < maxcy) {
    TRY(run_iteration(h, inner, &prof_ms, &prof_n, &prof_bytes));
    iter += 1;
    I.cycles += inner;
    rel = std::sqrt(h->h_res[0]) / bn;
    rmax = h->h_res[2];
    if (opts->record_history) h->history.push_back(opts->stop_rule == 1 ? rmax : rel);
    if (!std::isfinite(rel) || !std::isfinite(rmax) || rel > 1e8) { status = 2; break; }
    if (opts->stop_rule == 0 && rel <= opts->tol) status = 0;
    if (opts->stop_rule == 1 && rmax < opts->tol && iter > 1) status = 0;  // newsolv_mg.for:57
  }
  if (status != 2 && rmax > 10.0) status = 2;  // 'BIG RMAX!! STOP', newsolv_mg.for:65-75
  CU(cudaEventRecord(t1, h->st));
  CU(cudaEventSynchronize(t1));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  I.outer = iter;
  I.relres = rel;
  I.relres_block_max = rel;
  I.rmax = rmax;
  I.device_ms = ms;
  I.smoother_ms = prof_ms;
  I.smoother_launches = prof_n;
  I.smoother_bytes = prof_bytes;
  I.kernel_launches = h->kernels - k0;
  if (info) *info = I;
  TRY(check_device_error(h));
  if (status == 2) return fail(h, H3D_ERR_DIVERGED, "divergence not finite or rmax above 10");
  if (status != 0) return fail(h, H3D_ERR_NOT_CONVERGED, "not converged within maxcy cycles");
  return H3D_OK;
}

int h3d_mg_project(h3d_mg* h, double* const* p, double* const* u, double* const* v, double* const* w,
                   const double* const* ustar, const double* const* vstar, const double* const* wstar,
                   double dt, double alfapr, const h3d_solve_opts* opts, h3d_solve_info* info) {
  if (!h || !p || !u || !v || !w || !ustar || !vstar || !wstar || !opts) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_velocity(h));
  const int nb = (int)h->blocks.size();
  for (int ib = 0; ib < nb; ++ib) {
    const h3d_block_desc& d = h->blocks[ib];
    TRY(check_block_host_dims(h, d));
    const BlkLev& B = h->lev[1].geom.bl[ib];
    TRY(copy_field_3d(h, true, h->p64[h->pc], B, p[ib], d, true));
    TRY(copy_field_3d(h, true, h->vel[0], B, u[ib], d, true));
    TRY(copy_field_3d(h, true, h->vel[1], B, v[ib], d, true));
    TRY(copy_field_3d(h, true, h->vel[2], B, w[ib], d, true));
    TRY(copy_field_3d(h, true, h->vstar[0], B, const_cast<double*>(ustar[ib]), d, true));
    TRY(copy_field_3d(h, true, h->vstar[1], B, const_cast<double*>(vstar[ib]), d, true));
    TRY(copy_field_3d(h, true, h->vstar[2], B, const_cast<double*>(wstar[ib]), d, true));
  }
  int rc = h3d_mg_project_resident(h, dt, alfapr, opts, info);
  if (rc != H3D_OK && rc != H3D_ERR_NOT_CONVERGED) return rc;
  for (int ib = 0; ib < nb; ++ib) {
    const h3d_block_desc& d = h->blocks[ib];
    const BlkLev& B = h->lev[1].geom.bl[ib];
    TRY(copy_field_3d(h, false, h->p64[h->pc], B, p[ib], d, true));
    TRY(copy_field_3d(h, false, h->vel[0], B, u[ib], d, true));
    TRY(copy_field_3d(h, false, h->vel[1], B, v[ib], d, true));
    TRY(copy_field_3d(h, false, h->vel[2], B, w[ib], d, true));
  }
  CU(cudaStreamSynchronize(h->st));
  return rc;
}

// ---------------------------------------------------------- level hooks
static int level_ok(h3d_mg* h, int g) { return h && g >= 1 && g <= h->L; }

}  // extern "C"

// Copies a dense canonical block array (nz+2, ny+2, nx+2) of element type T
// to/from the padded device layout of block B.
template <typename T>
static int copy_canonical(h3d_mg* h, bool to_device, T* dev_level, const BlkLev& B, T* host) {
  cudaMemcpy3DParms p{};
  cudaPitchedPtr dptr = make_cudaPitchedPtr(dev_level + B.off, (size_t)B.sx * sizeof(T), B.nx + 2, B.ny + 2);
  cudaPitchedPtr hptr = make_cudaPitchedPtr(host, (size_t)(B.nx + 2) * sizeof(T), B.nx + 2, B.ny + 2);
  if (to_device) { p.srcPtr = hptr; p.dstPtr = dptr; p.kind = cudaMemcpyHostToDevice; }
  else { p.srcPtr = dptr; p.dstPtr = hptr; p.kind = cudaMemcpyDeviceToHost; }
  p.extent = make_cudaExtent((size_t)(B.nx + 2) * sizeof(T), B.ny + 2, B.nz + 2);
  CU(cudaMemcpy3DAsync(&p, h->st));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

extern "C" {

int h3d_mg_put_level(h3d_mg* h, int32_t g, int32_t field, int32_t ib, const double* a) {
  if (!level_ok(h, g) || !a || ib < 0 || ib >= (int)h->blocks.size() || field < 0 || field > 1) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->st));
  Level& V = h->lev[g];
  const BlkLev& B = V.geom.bl[ib];
  const size_t nb = (size_t)(B.nx + 2) * (B.ny + 2) * (B.nz + 2);
  std::vector<double> buf(nb, 0.0);
  if (field == 0) {
    std::memcpy(buf.data(), a, nb * 8);
  } else {
    for (int z = 1; z <= B.nz; ++z)
      for (int y = 1; y <= B.ny; ++y)
        for (int x = 1; x <= B.nx; ++x)
          buf[((size_t)z * (B.ny + 2) + y) * (B.nx + 2) + x] = a[((size_t)(z - 1) * B.ny + (y - 1)) * B.nx + (x - 1)];
  }
  const bool f32 = f32_level(h, g);
  if (f32) {
    std::vector<float> fb(buf.begin(), buf.end());
    TRY(copy_canonical<float>(h, true, field == 0 ? V.phi32[V.cur32] : V.rhs32, B, fb.data()));
    if (field == 0) V.zero32 = false;
  } else {
    TRY(copy_canonical<double>(h, true, field == 0 ? V.phi64[V.cur64] : V.rhs64, B, buf.data()));
    if (field == 0) V.zero64 = false;
  }
  return H3D_OK;
}

int h3d_mg_get_level(h3d_mg* h, int32_t g, int32_t field, int32_t ib, double* a) {
  if (!level_ok(h, g) || !a || ib < 0 || ib >= (int)h->blocks.size() || field < 0 || field > 1) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->st));
  Level& V = h->lev[g];
  const BlkLev& B = V.geom.bl[ib];
  const size_t nb = (size_t)(B.nx + 2) * (B.ny + 2) * (B.nz + 2);
  std::vector<double> buf(nb, 0.0);
  const bool f32 = f32_level(h, g);
  bool zero = f32 ? V.zero32 : V.zero64;
  if (!(field == 0 && zero)) {
    if (f32) {
      std::vector<float> fb(nb);
      TRY(copy_canonical<float>(h, false, field == 0 ? V.phi32[V.cur32] : V.rhs32, B, fb.data()));
      for (size_t q = 0; q < nb; ++q) buf[q] = fb[q];
    } else {
      TRY(copy_canonical<double>(h, false, field == 0 ? V.phi64[V.cur64] : V.rhs64, B, buf.data()));
    }
  }
  if (field == 0) {
    std::memcpy(a, buf.data(), nb * 8);
  } else {
    for (int z = 1; z <= B.nz; ++z)
      for (int y = 1; y <= B.ny; ++y)
        for (int x = 1; x <= B.nx; ++x)
          a[((size_t)(z - 1) * B.ny + (y - 1)) * B.nx + (x - 1)] = buf[((size_t)z * (B.ny + 2) + y) * (B.nx + 2) + x];
  }
  return H3D_OK;
}

int h3d_mg_mgrelax(h3d_mg* h, int32_t g, int32_t it) {
  if (!level_ok(h, g) || it < 0) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  Exec ex{h};
  TRY(ex.relax(g, it));
  CU(cudaStreamSynchronize(h->st));
  return check_device_error(h);
}

int h3d_mg_mgrestr(h3d_mg* h, int32_t g) {
  if (!level_ok(h, g) || g < 2) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  Exec ex{h};
  TRY(ex.restrict_to(g));
  // the reference zeroes the coarse iterate including ghosts (mgsolver.for:655-662)
  Level& C = h->lev[g];
  if (C.zero64 && C.phi64[0]) TRY(ex.materialize_zero64(g));
  if (C.zero32 && C.phi32[0]) TRY(ex.materialize_zero32(g));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_mgcorr(h3d_mg* h, int32_t g) {
  if (!level_ok(h, g) || g >= h->L) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  Exec ex{h};
  TRY(ex.correct(g));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

// Applies a halo table of `kind` out of place on the current iterate of level g.
static int apply_table_hook(h3d_mg* h, int g, int kind) {
  CU(cudaSetDevice(h->device));
  Level& V = h->lev[g];
  if (V.expr && kind == kHaloExchange) {  // exchangepp between blocks of different rdv
    if (!V.xe.built) TRY(upload_xfill(h, g, kHaloExchange, V.xe));
    Exec ex{h};
    const size_t n = (size_t)V.geom.n_elems;
    if (f32_level(h, g)) {
      if (V.zero32) TRY(ex.materialize_zero32(g));
      float* cur = V.phi32[V.cur32];
      float* nxt = V.phi32[1 - V.cur32];
      CU(cudaMemcpyAsync(nxt, cur, n * 4, cudaMemcpyDeviceToDevice, h->st));
      CU(run_xfill<float>(V, V.xe, nxt, cur, cur, false, h->st));
      V.cur32 = 1 - V.cur32;
    } else {
      if (V.zero64) TRY(ex.materialize_zero64(g));
      double* cur = V.phi64[V.cur64];
      double* nxt = V.phi64[1 - V.cur64];
      CU(cudaMemcpyAsync(nxt, cur, n * 8, cudaMemcpyDeviceToDevice, h->st));
      CU(run_xfill<double>(V, V.xe, nxt, cur, cur, false, h->st));
      V.cur64 = 1 - V.cur64;
    }
    CU(cudaStreamSynchronize(h->st));
    return H3D_OK;
  }
  Halo* H = kind == kHaloExchange ? &V.exch : &V.bound;
  if (!H->built) {
    std::vector<uint32_t> d, s;
    std::string err;
    int rc = build_halo_table(h->blocks, g, kind, true, d, s, &err);
    if (rc != H3D_OK) return fail(h, rc, err);
    TRY(upload_halo(h, *H, d, s));
    H->built = true;
  }
  const bool f32 = f32_level(h, g);
  const size_t n = (size_t)V.geom.n_elems;
  if (f32) {
    if (V.zero32) { Exec ex{h}; TRY(ex.materialize_zero32(g)); }
    float* cur = V.phi32[V.cur32];
    float* nxt = V.phi32[1 - V.cur32];
    CU(cudaMemcpyAsync(nxt, cur, n * 4, cudaMemcpyDeviceToDevice, h->st));
    if (H->n > 0) CU(launch_fill<float>(H->d_dst, H->d_src, H->n, nxt, cur, cur, false, h->st));
    V.cur32 = 1 - V.cur32;
  } else {
    if (V.zero64) { Exec ex{h}; TRY(ex.materialize_zero64(g)); }
    double* cur = V.phi64[V.cur64];
    double* nxt = V.phi64[1 - V.cur64];
    CU(cudaMemcpyAsync(nxt, cur, n * 8, cudaMemcpyDeviceToDevice, h->st));
    if (H->n > 0) CU(launch_fill<double>(H->d_dst, H->d_src, H->n, nxt, cur, cur, false, h->st));
    V.cur64 = 1 - V.cur64;
  }
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_mgbound(h3d_mg* h, int32_t g) {
  if (!level_ok(h, g)) return H3D_ERR_ARG;
  return apply_table_hook(h, g, kHaloBound);
}

int h3d_mg_exchangepp(h3d_mg* h, int32_t g) {
  if (!level_ok(h, g)) return H3D_ERR_ARG;
  return apply_table_hook(h, g, kHaloExchange);
}

int h3d_mg_vcycle(h3d_mg* h) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  Exec ex{h};
  TRY(ex.vcycle());
  CU(cudaStreamSynchronize(h->st));
  return check_device_error(h);
}

int h3d_mg_mgkcyc(h3d_mg* h, double* const* pp, const double* const* su) {
  if (!h || !pp || !su) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  TRY(ensure_coeffs(h));
  Level& V = h->lev[1];
  // pp (incl. one ghost layer) -> level-1 iterate, su -> level-1 rhs (mgsolver.for:239-266)
  for (int ib = 0; ib < (int)h->blocks.size(); ++ib) {
    if (h->mixed) {
      TRY(stage_in(h, 0, ib, pp[ib], h->p64[1 - h->pc], true));
      TRY(stage_in(h, 1, ib, su[ib], h->b64, false));
    } else {
      TRY(stage_in(h, 0, ib, pp[ib], V.phi64[V.cur64], true));
      TRY(stage_in(h, 1, ib, su[ib], V.rhs64, false));
    }
  }
  if (h->mixed) {
    CU(launch_convert_d2f(h->p64[1 - h->pc], V.phi32[V.cur32], V.geom.n_elems, h->st));
    CU(launch_convert_d2f(h->b64, V.rhs32, V.geom.n_elems, h->st));
    V.zero32 = false;
  } else {
    V.zero64 = false;
  }
  Exec ex{h};
  TRY(ex.vcycle());
  if (h->mixed) CU(launch_convert_f2d(V.phi32[V.cur32], h->p64[1 - h->pc], V.geom.n_elems, h->st));
  for (int ib = 0; ib < (int)h->blocks.size(); ++ib)
    TRY(stage_out(h, 0, ib, pp[ib], h->mixed ? h->p64[1 - h->pc] : V.phi64[V.cur64], true));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_sync(h3d_mg* h) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->st));
  return H3D_OK;
}

int h3d_mg_set_wait_limit(h3d_mg* h, int64_t clocks) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->st));
  CU(set_wait_clocks((long long)clocks));
  return H3D_OK;
}

int h3d_mg_wait_probe(h3d_mg* h) {
  if (!h) return H3D_ERR_ARG;
  CU(cudaSetDevice(h->device));
  CU(launch_wait_probe(h->d_err, h->st));
  CU(cudaStreamSynchronize(h->st));
  return check_device_error(h);
}

int h3d_mg_set_profiling(h3d_mg* h, int32_t on) {
  if (!h) return H3D_ERR_ARG;
  h->profiling = on != 0;
  return H3D_OK;
}

int h3d_mg_set_smoother(h3d_mg* h, int32_t g, int32_t variant, int32_t zchunk) {
  if (!level_ok(h, g) || variant < 0 || variant >= num_tile_shapes() || zchunk < 1) return H3D_ERR_ARG;
  Level& V = h->lev[g];
  if (!variant_fits(V, variant)) return fail(h, H3D_ERR_ARG, "smoother variant does not fit this level");
  CU(cudaSetDevice(h->device));
  TRY(build_tiles(h, V, variant, zchunk));
  h->graphs.clear();  // captured graphs refer to the old tiles
  return H3D_OK;
}

int h3d_mg_get_smoother(h3d_mg* h, int32_t g, int32_t* variant, int32_t* zchunk, int32_t* nvariants) {
  if (!level_ok(h, g)) return H3D_ERR_ARG;
  if (variant) *variant = h->lev[g].variant;
  if (zchunk) *zchunk = h->lev[g].zc;
  if (nvariants) *nvariants = num_tile_shapes();
  return H3D_OK;
}

int h3d_mg_set_restriction(h3d_mg* h, int32_t g, int32_t variant, int32_t zchunk) {
  if (!level_ok(h, g) || g < 2 || variant < 0 || variant >= num_restrict_shapes() || zchunk < 1)
    return H3D_ERR_ARG;
  Level& F = h->lev[g - 1];
  Level& C = h->lev[g];
  RestrictShape r = restrict_shape(variant);
  int nxm = 0;
  for (const auto& B : C.geom.bl) nxm = std::max(nxm, B.nx);
  if (r.tpr * r.cpx < nxm || (r.tma && (!F.tma_ok || !F.d_rmaps)))
    return fail(h, H3D_ERR_ARG, "restriction variant does not fit this level");
  CU(cudaSetDevice(h->device));
  std::vector<Tile> t = row_tiles(C.geom, r.tyc, zchunk);
  TRY(upload_tiles(h, &C.d_rtiles, &C.rtiles_cap, t));
  C.nrtiles = (int)t.size();
  C.rvariant = variant;
  C.rzc = zchunk;
  h->graphs.clear();  // captured graphs refer to the old tiles
  return H3D_OK;
}

int h3d_mg_get_restriction(h3d_mg* h, int32_t g, int32_t* variant, int32_t* zchunk, int32_t* nvariants) {
  if (!level_ok(h, g) || g < 2) return H3D_ERR_ARG;
  if (variant) *variant = h->lev[g].rvariant;
  if (zchunk) *zchunk = h->lev[g].rzc;
  if (nvariants) *nvariants = num_restrict_shapes();
  return H3D_OK;
}

int h3d_mg_smoother_bytes(h3d_mg* h, double* bytes) {
  if (!h || !bytes) return H3D_ERR_ARG;
  *bytes = h->lev[1].sweep_bytes;
  return H3D_OK;
}

}  // extern "C"
