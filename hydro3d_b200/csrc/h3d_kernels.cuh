// Device kernels of the multigrid V-cycle (declarations of the launchers).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "h3d_internal.h"

namespace h3d {

// Cell launch table: CTAs of a cell kernel are assigned to blocks by prefix;
// cta_start[b] is the first CTA of block b, cta_start[nb] the total.
struct CellTab {
  const int* cta_start;  // device
  int nb;
  int ncta;
};

// Row table: one warp per row; start[b] is the first row of block b,
// start[nb] == nrows.
struct RowTab {
  const int* start;  // device
  int nb;
  int nrows;
};

// Smoother tile shapes the runtime can choose (autotuned per level).  Row
// shapes (rows == true) span whole rows: usable when every block's nx is even
// and <= tx.
struct TileShape {
  int tx, ty, nt;
  bool rows;
  int tpr, cp;
  int tma;   // 0 plain loads; 1 iterate planes staged by TMA; 2 iterate and right-hand side by TMA;
             // 3 as 2, vectorised (FP32, constant coefficients, nx a multiple of 4 and <= tx)
  int alt;   // for TMA shapes: the equivalent row shape (used for zero sources)
};
// TMA box heights (TY+4) are one of these; tensor maps are built per height.
constexpr int kNumTmaTy = 5;
int tma_ty_index(int ty);  // 0,1,2,3,4 for TY = 4, 8, 16, 32, 15; -1 otherwise
constexpr int kDefectCtas = 148 * 4;  // CTAs (and partial sums) of the defect kernel
int defect_grid(int nrows);
// Sets the dynamic shared-memory limits of the row-tile smoothers (call once
// per device before any launch or capture).
cudaError_t init_kernel_attributes();
cudaError_t init_kernel_attributes_2();  // restriction tiles

// Tile restriction shapes: TPR threads per coarse row, CPX coarse cells per
// thread (coarse nx <= TPR*CPX), TYC coarse rows per CTA; tma: fine planes
// staged by TMA (needs the fine level's restriction tensor maps for TYC).
struct RestrictShape {
  int tpr, cpx, tyc, tma;
};
int num_restrict_shapes();
RestrictShape restrict_shape(int v);
constexpr int kNumRTmaTyc = 2;
int rtma_tyc_index(int tyc);  // 0, 1 for TYC = 4, 8; -1 otherwise
// pmaps: tensor maps of the fine iterate (box 2*TYC+2 fine rows); rmaps: of the
// fine right-hand side (box 2*TYC rows); both only for TMA shapes.
template <typename T>
cudaError_t launch_restrict_tile(int variant, bool var, bool zero_phi, const BlkLev* fine, const BlkLev* coarse,
                                 const Tile* tiles, int ntiles, int zc, const T* phi, const T* rhs, T* rhs_c,
                                 const T* fx, const T* fy, const T* fz, const CUtensorMap* pmaps,
                                 const CUtensorMap* rmaps, int* err, cudaStream_t st);

// Moves the region (ex, ey, ez) starting at canonical (g0, g0, g0) of one
// block between a whole host block array staged on the device (dims tx, ty,
// tz, pl ghost layers) and the padded device layout (block base dev).
cudaError_t launch_stage(bool to_device, double* stg, int tx, int ty, int pl, int g0, int ex, int ey, int ez,
                         double* dev, int sx, long long sxy, cudaStream_t st);

int num_tile_shapes();
TileShape tile_shape(int variant);

// One out-of-place red-black sweep (both colours) of every block of a level:
// dst = sweep(src).  zero_src: src is identically zero (not read).
// maps: tensor maps of src for every block (TMA variants); rmaps: tensor maps
// of rhs (variants that stage it); err: device flag set when a bounded wait
// gives up.
// push: per block, six element offsets (faces W, E, S, N, B, T; kNoPush: none)
// from a face cell to the ghost cell it is the source of; the register-window
// sweeps store their new face values there too (others reject a push table).
constexpr long long kNoPush = (long long)(~0ull >> 1);
bool rbgs_pushes(int variant, bool var, bool f32);
template <typename T>
cudaError_t launch_rbgs(int variant, bool var, bool zero_src, const BlkLev* bl, const Tile* tiles,
                        int ntiles, int zc, const CUtensorMap* maps, const CUtensorMap* rmaps, int* err,
                        const T* src, T* dst,
                        const T* rhs, const T* fx, const T* fy,
                        const T* fz, const long long* push, float om, cudaStream_t st);

constexpr int kSmallLevelBlocks = 64;  // block descriptors the fused small-level kernel caches
// `sweeps` red-black sweeps of a small level, each followed by its ghost fill,
// in place in one CTA (see k_relax_small).  start: flat interior index of
// each block's first cell (nb+1 entries); the fill table must read interior
// cells only.
// The coarse end of a V-cycle in one CTA (k_coarse_tail), every tail level
// in shared memory in a compact layout: per tail level its block tables
// (global layout for loads and stores; compact layout with the rhs base of
// each block in .pad), cell tables, compact fill table, global buffers and
// the byte offsets of its arrays in the shared arena (-1: absent).
struct TailLevel {
  const BlkLev* gbl;
  const BlkLev* cbl;
  const unsigned long long* cells;   // interior cells, red (x+y+z odd) first
  const unsigned long long* ghosts;  // ghost cells of the padded blocks
  const uint32_t* fdst;              // sweep fill table, compact indices (cluster tail: own block)
  const uint32_t* fsrc;              // (cluster tail: source rank << 24 | compact index in its block)
  const int* fstart;                 // cluster tail: fill entries of block b are fstart[b] .. fstart[b+1]-1
  int nb, nint, nred, nghost, npad, nfill;
  float* phi32[2];
  float* rhs32;
  double* phi64[2];
  double* rhs64;
  int s_phi32, s_rhs32, s_phi64, s_rhs64;
  int s_cells, s_fill;  // cluster tail: arena offsets of the staged cell tables and this block's fill pairs
  const double* dense;  // coarsest level solved directly: its pseudo-inverse, dense_n x dense_n, row-major
  int dense_n;
  float om;             // over-relaxation of the level's FP32 sweeps (1: Gauss-Seidel)
  int rb_global;        // 1: a ghost fill after each colour (red-black order across block faces)
};
enum TailKind {
  kTailRelax = 0,
  kTailRestrict = 1,
  kTailProlong = 2,
  kTailRhsF2D = 3,
  kTailPhiD2F = 4,
  kTailLoadRhs = 5,
  kTailStore = 6,
  kTailDense = 7  // cluster tail: phi = P rhs on the coarsest level (FP64), then its fill
};
constexpr int kDenseMaxCells = 512;  // largest coarsest level solved by its pseudo-inverse
struct TailOp {
  int kind;
  int f64;     // the op runs in FP64
  int fine;    // relax / conversions / load / store: the level; restrict / prolong: the fine level
  int coarse;  // restrict / prolong: the coarse level
  int sweeps;  // relax: sweeps; prolong: arena offset of the ghost scratch
  int zero;    // relax: zero the iterate first; restrict / prolong: the fine iterate is zero
};
constexpr int kTailMaxLevels = 16;  // curmask holds two bits a level
constexpr int kTailSmemBytes = 212 * 1024;  // shared arena of the tail (+ 12 KB of block tables)
// Cell entry of the tail tables: compact index (24 bits), x, y, z (8 bits each), block (6 bits).
inline unsigned long long tail_cell(long long i, int x, int y, int z, int b) {
  return (unsigned long long)i | ((unsigned long long)x << 24) | ((unsigned long long)y << 32) |
         ((unsigned long long)z << 40) | ((unsigned long long)b << 48);
}
cudaError_t launch_coarse_tail(const TailLevel* lv, const TailOp* ops, int nops, unsigned curmask, int smem_bytes,
                               cudaStream_t st);
// The same program as one cluster of nb CTAs (nb <= 16), CTA b holding block b
// of every tail level (all blocks of a level the same size).
constexpr int kClusterTailThreads = 512;
constexpr int kClusterTailMaxBlocks = 16;
int coarse_cluster_fits(int nb, int smem_bytes);  // clusters that can be resident at once (0: none)
constexpr int kClusterTailMaxOps = 160;
cudaError_t launch_coarse_cluster(int nb, const TailLevel* lv, int nlev, const TailOp* ops, int nops,
                                  unsigned curmask, int smem_bytes, cudaStream_t st);

// First red-black sweep from a zero iterate of an FP32 constant-coefficient
// level (every block's nx a multiple of 4, at most 1024): tiles (block, y0 =
// first row, z0 = first plane) of 256 / (nx/4) rows and zc planes.
cudaError_t launch_rbgs_zero32(const BlkLev* bl, const Tile* tiles, int ntiles, int zc, const float* rhs, float* dst,
                               const long long* push, float om, cudaStream_t st);
// Lexicographic Gauss-Seidel (itrsch 1) or line-TDMA (itrsch 2) sweep of
// every block of a level, one CTA per block (bit-exact wavefront orderings
// of mgsolver.for:407-549); acoef: level-sized scratch of the TDMA.
template <typename T>
cudaError_t launch_seq_smoother(int itrsch, bool var, bool zero, const BlkLev* bl, int nb, const T* src, T* dst,
                                const T* rhs, T* acoef, const T* fx, const T* fy, const T* fz, cudaStream_t st);
template <typename T>
cudaError_t launch_relax_small(bool var, const BlkLev* bl, const int* start, int nb, T* phi, const T* rhs,
                               const T* fx, const T* fy, const T* fz, const uint32_t* fdst, const uint32_t* fsrc,
                               int nfill, int sweeps, bool zero, long long nelems, float om, bool rb,
                               cudaStream_t st);

// Ghost gather: out[dst[e]] = (src[e] & old) ? old[src] : cur[src].
template <typename T>
cudaError_t launch_fill(const uint32_t* dsts, const uint32_t* srcs, int64_t n, T* out, const T* cur,
                        const T* old, bool zero_old, cudaStream_t st);

// Red updates of the red cells next to block faces, stored at the ghost cells
// that show them to other blocks (FP32, before a sweep; see k_red_ahead).
cudaError_t launch_red_ahead(bool var, const uint32_t* dst, const uint32_t* src, const int* info, int64_t n, int nb,
                             const BlkLev* bl, float* phi, const float* rhs, const float* fx, const float* fy,
                             const float* fz, float om, cudaStream_t st);

// Residual of the fine level and 8-cell average into the coarse rhs
// (mgrestr, mgsolver.for:693-756).  zero_phi: fine iterate is zero.
template <typename T>
cudaError_t launch_restrict(bool var, bool zero_phi, const BlkLev* fine, const BlkLev* coarse, RowTab rt,
                            const T* phi, const T* rhs, T* rhs_c, const T* fx, const T* fy, const T* fz,
                            cudaStream_t st);

// Trilinear correction (mgcorr, mgsolver.for:828-896) with the following
// mgbound fused: out = old + P(coarse), evaluated at the mgbound source.
template <typename T>
cudaError_t launch_prolong(bool zero_old, const BlkLev* fine, const BlkLev* coarse, RowTab rt,
                           const T* phi_c, const T* old, T* out, cudaStream_t st);
// Same, tiled: tiles (b, 0, 0, 2m) of fine plane pairs (2m, 2m+1), ghost
// planes included; needs every block's nx a multiple of 16/sizeof(T) and
// ny, nz even.
constexpr int kProlongRows = 32;  // rows of a tile of the tiled defect
template <typename T>
cudaError_t launch_prolong_vec(bool zero_old, const BlkLev* fine, const BlkLev* coarse, const Tile* tiles, int ntiles,
                               const T* phi_c, const T* old, T* out, cudaStream_t st);

// Tiled defect (constant coefficients, nx even): tiles of kProlongRows rows of
// one plane (the level's prolongation tiles), one CTA and partial sum each.
template <typename TE, typename TR>
cudaError_t launch_defect_vec(const BlkLev* bl, const Tile* tiles, int ntiles, const double* p, const TE* e,
                              double* p_next, const double* b, TR* rhs_out, double mean_b, double rscale,
                              double* partials, int grid, cudaStream_t st);

// The same defect as a z march (constant coefficients, nx even, nx <= 64 gp):
// tiles of defect_march_rows() interior rows of one block over zc planes from
// z0, one CTA and partial sum each; gp = 1, 2 or 4 pairs of cells per lane.
template <typename TE, typename TR>
cudaError_t launch_defect_march(int gp, const BlkLev* bl, const Tile* tiles, int ntiles, int zc, const double* p,
                                const TE* e, double* p_next, const double* b, TR* rhs_out, double mean_b,
                                double rscale, double* partials, cudaStream_t st);
int defect_march_rows();

// Level-1 FP64 defect: pn = p + e (all cells, when e != null), r = b - A pn on
// the interior, rhs_out = r - mean_b (as TR), per-CTA partial sums
// {sum r^2, sum b^2, max |r|*rscale, sum r} into partials[4*cta]; rscale < 0
// stands for each block's own cell volume dv.
template <typename TE, typename TR>
cudaError_t launch_defect(bool var, const BlkLev* bl, RowTab rt, const double* p, const TE* e,
                          double* p_next, const double* b, TR* rhs_out, double mean_b, double rscale,
                          const double* fx, const double* fy, const double* fz, double* partials,
                          cudaStream_t st);
// Deterministic reduction of n partial quadruples into out[4].
cudaError_t launch_reduce4(const double* partials, int n, double* out, cudaStream_t st);
// Per-block sums: out[4b..4b+3] from partials start[b] .. start[b+1]-1.
cudaError_t launch_reduce4_blocks(const double* partials, const int* start, int nb, double* out, cudaStream_t st);

// Interior sum of a level-1 field (per-CTA partials, reduce with launch_reduce4).
cudaError_t launch_sum_interior(const BlkLev* bl, RowTab rt, const double* a, double* partials, int* nparts,
                                cudaStream_t st);
// a -= s on every cell (incl. ghosts); s read from device memory.
cudaError_t launch_shift(double* a, int64_t n, const double* s, double scale, cudaStream_t st);

// Precision conversions of whole level arrays.
cudaError_t launch_convert_d2f(const double* a, float* b, int64_t n, cudaStream_t st);
cudaError_t launch_convert_f2d(const float* a, double* b, int64_t n, cudaStream_t st);

// L_LSM coefficients (mgsolver.for:72-184): dens of the finer level -> dens of
// level g (8-cell average), and the face coefficient arrays of level g.
cudaError_t launch_dens_restrict(const BlkLev* fine, const BlkLev* coarse, CellTab ct, const double* df,
                                 double* dc, cudaStream_t st);
cudaError_t launch_face_coef(const BlkLev* bl, CellTab ct, const double* dens, const double* h3 /*per block dx,dy,dz*/,
                             double* fx, double* fy, double* fz, cudaStream_t st);

// Limit of every bounded mbarrier wait on the current device, in SM clocks
// (<= 0: the default 2^26).
cudaError_t set_wait_clocks(long long clocks);
// One bounded wait on an mbarrier nothing arrives at (sets *err when it gives up).
cudaError_t launch_wait_probe(int* err, cudaStream_t st);

// Face-sum coarse coefficients of level g from those of level g-1 (L_LSM,
// coarse_op 1): a coarse face = (sum of its four fine faces) / 16.
cudaError_t launch_face_coef_sum(const BlkLev* fine, const BlkLev* coarse, CellTab ct, const double* ffx,
                                 const double* ffy, const double* ffz, double* cfx, double* cfy, double* cfz,
                                 cudaStream_t st);

// `sweeps` in-place red-black sweeps of a level whose ghost fill is
// block-local, one CTA per block; fstart: fill entries of each block (the
// table sorted by block, nb + 1 entries).
template <typename T>
cudaError_t launch_relax_blocks(bool var, const BlkLev* bl, int nb, const int* fstart, T* phi, const T* rhs,
                                const T* fx, const T* fy, const T* fz, const uint32_t* fdst, const uint32_t* fsrc,
                                int sweeps, bool zero, float om, cudaStream_t st);

// Stone's SIP (sipsol.for) on level 1: factor arrays and the residual
// (level-1 layout, zero outside the interior).
struct SipArrays {
  double *lb, *lw, *ls, *lpr, *un, *ue, *ut, *res;
};
cudaError_t launch_sip_factor(const BlkLev* bl, int nb, SipArrays a, cudaStream_t st);
// One sweep of every block on fi with rhs su; partials[4b] = sum |res| of block b.
cudaError_t launch_sip_sweep(const BlkLev* bl, int nb, SipArrays a, double* fi, const double* su, double* partials,
                             cudaStream_t st);
// a[dst[e]] = a[src[e]].
cudaError_t launch_gather1(const uint32_t* dst, const uint32_t* src, int64_t n, double* a, cudaStream_t st);

// The projection on level 1 (press.for:2-144, newsolv_mg.for:39-49).
// calvel: u, v, w from ustar, vstar, wstar and p (dtal = dt*alfapr; dens read
// for L_LSM only).
cudaError_t launch_calvel(bool lsm, const BlkLev* bl, RowTab interior_rows, const double* h3, const double* p,
                          const double* dens, const double* us, const double* vs, const double* ws, double* u,
                          double* v, double* w, double dtal, cudaStream_t st);
// a_c[dst[e]] = a_c[src[e]] for the three arrays (velocity face ghosts).
cudaError_t launch_gather3(const uint32_t* dst, const uint32_t* src, int64_t n, double* a0, double* a1, double* a2,
                           cudaStream_t st);
// calmas: su into bout (FP64) and rhs_out (TR); partials {sum su^2, 0, rmax,
// sum su} per CTA (*nparts of them, reduce with launch_reduce4).
template <typename TR>
cudaError_t launch_calmas(bool lsm, const BlkLev* bl, RowTab interior_rows, const double* h3, const double* u,
                          const double* v, const double* w, double dt, double* bout, TR* rhs_out, double* partials,
                          int* nparts, cudaStream_t st);
// p += e on every cell of every row (ghost layer included).
template <typename TE>
cudaError_t launch_padd(const BlkLev* bl, RowTab all_rows, double* p, const TE* e, cudaStream_t st);

// Local mesh refinement.  Expression fill of a level (see ExprTable): one
// launch per node depth (depth_start: host array of ndepth + 1 offsets), then
// the ghost writes out[dst[e]] = ref(src[e]).  cur: current values (may be
// out), old: pre-fill values (zero_old: all zero), scratch: node values.
template <typename T>
cudaError_t launch_expr_fill(const uint32_t* nodes, const int64_t* depth_start, int ndepth, const uint32_t* dst,
                             const uint32_t* src, int64_t nw, T* out, const T* cur, const T* old, bool zero_old,
                             T* scratch, cudaStream_t st);
// mgrestr for the listed blocks past their last level (glevel > ngrid,
// mgsolver.for:724-737): the coarse rhs is the fine residual, cell for cell.
template <typename T>
cudaError_t launch_restrict_same(bool zero_phi, const BlkLev* fine, const BlkLev* coarse, const int* blist, int nbl,
                                 int max_cells, const T* phi, const T* rhs, T* rhs_c, cudaStream_t st);
// mgcorr for the listed blocks whose coarser level is the same size
// (glevel >= ngrid, mgsolver.for:812-824): out = old + coarse on every cell,
// with the following mgbound fused (ghosts of wall faces read their source).
template <typename T>
cudaError_t launch_prolong_same(bool zero_old, const BlkLev* fine, const BlkLev* coarse, const int* blist, int nbl,
                                int max_cells, const T* phi_c, const T* old, T* out, cudaStream_t st);

}  // namespace h3d
