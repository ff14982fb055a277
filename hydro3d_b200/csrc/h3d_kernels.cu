// sm_100a kernels of the multigrid V-cycle.
//
// All FP64 arithmetic follows the reference's operand order (mgsolver.for)
// and the library is compiled with --fmad=false, so the FP64 path reproduces
// the reference arithmetic bit for bit.  Every kernel is memory bound (a
// 7-point stencil is not a contraction; no tensor cores are used).
#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include <type_traits>

#include <cooperative_groups.h>

#include "h3d_kernels.cuh"

namespace h3d {

namespace {

// Programmatic dependent launch (opt-in, H3D_PDL=1 in the environment): every
// kernel lets the next one on the stream start launching at once
// (griddepcontrol.launch_dependents) and waits for its predecessors to
// complete (griddepcontrol.wait) before it touches data they write.  Both are
// no-ops for a kernel launched without the attribute.  For every launch it
// measured 60.1 ms against 56.1 ms without on the 33.5M-cell solve (the
// early launched grids hold SM resources the running ones need).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// Over-relaxed red-black update of the FP32 inner solve: x + om (gs - x), om
// the handle's over-relaxation factor (1: Gauss-Seidel up to rounding).  The
// FP64 sweeps keep the reference's update.
__device__ __forceinline__ float sorf(float old, float gs, float om) { return fmaf(om, gs - old, old); }

// Launch policy (H3D_PDL): "1" every kernel, "0" none; by default only a
// kernel of at most kPdlGrid CTAs that follows one of at most kPdlGrid CTAs
// on the same host thread.  Such a predecessor runs in a single wave, so the
// early-launched grid only takes SM slots that the predecessor leaves idle,
// while the launch latency of the chains of small kernels of the coarse
// levels is hidden.
constexpr long long kPdlGrid = 2 * 148;
static int pdl_mode() {
  static const int m = [] {
    const char* v = std::getenv("H3D_PDL");
    if (v && v[0] == '1') return 1;
    if (v && v[0] == '0') return 0;
    return 2;
  }();
  return m;
}
static thread_local long long g_prev_grid = 1LL << 40;

template <typename... KArgs, typename... Args>
static cudaError_t pdl_launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  const long long n = (long long)grid.x * grid.y * grid.z;
  const int mode = pdl_mode();
  cfg.numAttrs = (mode == 1 || (mode == 2 && n <= kPdlGrid && g_prev_grid <= kPdlGrid)) ? 1 : 0;
  g_prev_grid = n;
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

__device__ __forceinline__ int find_block(const int* __restrict__ start, int nb, int cta) {
  int lo = 0, hi = nb;  // start[lo] <= cta < start[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(start + mid) <= cta) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Bounds-checked debug builds (-DH3D_BOUNDS_CHECK): accesses of the tile
// kernels are checked against their block / shared-memory extents; the first
// violation (kernel id, block, index, limit) is recorded and the access
// skipped, so a wrong index shows up as a record instead of a fault.
#ifdef H3D_BOUNDS_CHECK
__device__ unsigned long long g_h3d_bad[4];
__device__ __noinline__ bool h3d_oob(int kid, int b, long long idx, long long lim) {
  if (idx >= 0 && idx < lim) return false;
  if (atomicCAS(&g_h3d_bad[0], 0ull, (unsigned long long)(kid + 1)) == 0ull) {
    g_h3d_bad[1] = (unsigned long long)b;
    g_h3d_bad[2] = (unsigned long long)idx;
    g_h3d_bad[3] = (unsigned long long)lim;
  }
  return true;
}
#define H3D_IN(kid, b, idx, lim) (!h3d_oob((kid), (b), (long long)(idx), (long long)(lim)))
#else
#define H3D_IN(kid, b, idx, lim) true
#endif

template <typename T>
struct Coef {
  T aw, ae, as, an, ab, at;
};

// Face coefficients of interior cell (x,y,z) (mgsolver.for:186-205).
template <typename T, bool VAR>
__device__ __forceinline__ Coef<T> cell_coef(const BlkLev& B, int x, int y, int z, long long i, const T* fx,
                                             const T* fy, const T* fz) {
  Coef<T> c;
  if (VAR) {
    c.aw = fx[i - 1];
    c.ae = fx[i];
    c.as = fy[i - B.sx];
    c.an = fy[i];
    c.ab = fz[i - B.sxy];
    c.at = fz[i];
  } else {
    const T ax = (T)B.ax, ay = (T)B.ay, az = (T)B.az;
    const int ph = B.phys;
    c.aw = (x == 1 && (ph & 1)) ? T(0) : ax;
    c.ae = (x == B.nx && (ph & 2)) ? T(0) : ax;
    c.as = (y == 1 && (ph & 4)) ? T(0) : ay;
    c.an = (y == B.ny && (ph & 8)) ? T(0) : ay;
    c.ab = (z == 1 && (ph & 16)) ? T(0) : az;
    c.at = (z == B.nz && (ph & 32)) ? T(0) : az;
  }
  return c;
}

template <typename T>
__device__ __forceinline__ T coef_ap(const Coef<T>& c) {
  return -(c.aw + c.ae + c.as + c.an + c.ab + c.at);  // -1.0*(...), mgsolver.for:207-210
}

// Gauss-Seidel update division: IEEE division in FP64 (the reference's
// arithmetic); the FP32 inner solve uses the 2-ulp reciprocal division.
__device__ __forceinline__ double gs_div(double a, double b) { return a / b; }
__device__ __forceinline__ float gs_div(float a, float b) { return __fdividef(a, b); }

// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel sweep (mgrelax, mg_itrsch=3, mgsolver.for:551-605).
//
// Colour = MOD(i+j+k,2) of the reference's 1-based ghost-inclusive indices,
// i.e. red (first pass) <=> x+y+z odd in 0-based ghost-inclusive coordinates.
// The sweep is out of place: every CTA reads the previous iterate `src` and
// writes `dst`, so tiles can overlap without ordering between CTAs.  A CTA
// owns a TX x TY column of one block and marches a z range through a ring of
// four shared-memory planes: at step z it stages plane z+1, updates the red
// cells of plane z on the tile plus a one-cell ring (their old black
// neighbours are in the two-cell staged halo), then updates the black cells
// of plane z-1 from the new red values and stores plane z-1.  Ghost cells are
// never updated inside a sweep, exactly like the reference, where they change
// only in the mgbound/exchangepp call after the whole sweep.
template <typename T, int TX, int TY, int NT, bool VAR, bool ZERO>
__global__ void __launch_bounds__(NT) k_rbgs(const BlkLev* __restrict__ bls, const Tile* __restrict__ tiles,
                                             int zc, const T* __restrict__ src, T* __restrict__ dst,
                                             const T* __restrict__ rhs, const T* __restrict__ fx,
                                             const T* __restrict__ fy, const T* __restrict__ fz, float om) {
  pdl_trigger();
  pdl_wait();
  constexpr int RX = TX + 4, RY = TY + 4, RN = RX * RY;
  constexpr int R1X = TX + 2, R1N = (TX + 2) * (TY + 2);
  __shared__ T ring[4][RN];
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sx = B.sx, sxy = B.sxy;
  const T* __restrict__ S = src + B.off;
  T* __restrict__ D = dst + B.off;
  const T* __restrict__ R = rhs + B.off;
  const T* FX = VAR ? fx + B.off : nullptr;
  const T* FY = VAR ? fy + B.off : nullptr;
  const T* FZ = VAR ? fz + B.off : nullptr;
  const int x0 = t.x0, y0 = t.y0, zs = t.z0;
  const int ze = min(zs + zc - 1, nz);
  const int zlo = max(zs - 1, 1), zhi = min(ze + 1, nz);

  auto stage = [&](int z) {
    T* P = ring[z & 3];
    const T* Sz = S + (long long)z * sxy;
    for (int q = threadIdx.x; q < RN; q += NT) {
      int ly = q / RX, lx = q - ly * RX;
      int x = x0 - 2 + lx, y = y0 - 2 + ly;
      T v = T(0);
      if (!ZERO && x >= 0 && x <= nx + 1 && y >= 0 && y <= ny + 1) v = Sz[y * sx + x];
      P[q] = v;
    }
  };
  auto red = [&](int z) {
    T* P = ring[z & 3];
    const T* Pm = ring[(z - 1) & 3];
    const T* Pp = ring[(z + 1) & 3];
    for (int q = threadIdx.x; q < R1N; q += NT) {
      int ly = q / R1X, lx = q - ly * R1X;
      int x = x0 - 1 + lx, y = y0 - 1 + ly;
      if (x < 1 || x > nx || y < 1 || y > ny || ((x + y + z) & 1) == 0) continue;
      int s = (ly + 1) * RX + lx + 1;
      long long i = (long long)z * sxy + y * sx + x;
      Coef<T> c = cell_coef<T, VAR>(B, x, y, z, i, FX, FY, FZ);
      T ap = coef_ap(c);
      const T gv = gs_div(R[i] - (c.aw * P[s - 1] + c.ae * P[s + 1] + c.as * P[s - RX] + c.an * P[s + RX] +
                                  c.ab * Pm[s] + c.at * Pp[s]),
                          ap);
      if constexpr (sizeof(T) == 4) P[s] = sorf(P[s], gv, om);
      else P[s] = gv;
    }
  };
  auto black_store = [&](int z) {
    const T* P = ring[z & 3];
    const T* Pm = ring[(z - 1) & 3];
    const T* Pp = ring[(z + 1) & 3];
    T* Dz = D + (long long)z * sxy;
    for (int q = threadIdx.x; q < TX * TY; q += NT) {
      int ly = q / TX, lx = q - ly * TX;
      int x = x0 + lx, y = y0 + ly;
      if (x > nx || y > ny) continue;
      int s = (ly + 2) * RX + lx + 2;
      long long i = (long long)z * sxy + y * sx + x;
      T v;
      if ((x + y + z) & 1) {
        v = P[s];  // red, updated at the previous step
      } else {
        Coef<T> c = cell_coef<T, VAR>(B, x, y, z, i, FX, FY, FZ);
        T ap = coef_ap(c);
        v = gs_div(R[i] - (c.aw * P[s - 1] + c.ae * P[s + 1] + c.as * P[s - RX] + c.an * P[s + RX] +
                           c.ab * Pm[s] + c.at * Pp[s]),
                   ap);
        if constexpr (sizeof(T) == 4) v = sorf(P[s], v, om);
      }
      Dz[y * sx + x] = v;
    }
  };

  stage(zlo - 1);
  stage(zlo);
  for (int z = zlo; z <= zhi; ++z) {
    stage(z + 1);
    __syncthreads();
    red(z);
    __syncthreads();
    if (z - 1 >= zs && z - 1 <= ze) black_store(z - 1);
    __syncthreads();
  }
  if (ze == nz) black_store(nz);
}


// ---------------------------------------------------------------------------
// First red-black sweep from a zero iterate (FP32, constant coefficients) as
// a stencil on the right-hand side.  With a zero source every red cell only
// sees black neighbours that are still zero, so red = rhs * (1/ap); a black
// cell sees red neighbours, each rhs_nb * (1/ap_nb) inside the block and zero
// outside it (the ghosts of a zero iterate).  These are the exact FP32
// operations of the TMA window sweep in its zero-source mode (same products,
// same fused multiply-add chain), evaluated without its plane ring and
// per-plane barriers: a thread owns one 4-cell group of one row and marches a
// chunk of planes, keeping the group's right-hand side of planes z-1, z, z+1
// in registers; rows y+-1 and the two cells beside the group come from L1.
// 1/ap of a cell depends only on which wall faces it touches: a 64-entry
// table per CTA.  Ghost pushes as in the window sweep.
__global__ void __launch_bounds__(256, 3) k_rbgs_zero32(const BlkLev* __restrict__ bls, const Tile* __restrict__ tiles,
                                                     int zc, const float* __restrict__ rhs, float* __restrict__ dst,
                                                     const long long* __restrict__ push, float om) {
  pdl_trigger();
  __shared__ float ivtab[64];
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const int nx = B.nx, ny = B.ny, nz = B.nz, ph = B.phys;
  const float ax = (float)B.ax, ay = (float)B.ay, az = (float)B.az;
  if (threadIdx.x < 64) {
    const int m = threadIdx.x;
    const float aw = (m & 1) ? 0.f : ax, ae = (m & 2) ? 0.f : ax, as = (m & 4) ? 0.f : ay, an = (m & 8) ? 0.f : ay,
                ab = (m & 16) ? 0.f : az, at = (m & 32) ? 0.f : az;
    ivtab[m] = 1.f / (-(aw + ae + as + an + ab + at));
  }
  __syncthreads();
  pdl_wait();
  const int G = nx >> 2;           // groups per row
  const int rows = blockDim.x / G;  // rows of this tile
  const int r = threadIdx.x / G, g = threadIdx.x - r * G;
  const int y = t.y0 + r;
  if (r >= rows || y > ny) return;
  const int x0 = 1 + 4 * g;
  const long long sx = B.sx, sxy = B.sxy;
  const float* __restrict__ R = rhs + B.off;
  float* __restrict__ D = dst + B.off;
  const int zs = t.z0, ze = min(t.z0 + zc - 1, nz);
  // wall mask of a cell (only faces that are physical walls count)
  auto wmask = [&](int x, int yy, int z) {
    return ph & ((x == 1 ? 1 : 0) | (x == nx ? 2 : 0) | (yy == 1 ? 4 : 0) | (yy == ny ? 8 : 0) | (z == 1 ? 16 : 0) |
                 (z == nz ? 32 : 0));
  };
  long long pd[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) pd[f] = push ? __ldg(push + 6 * t.b + f) : kNoPush;
  const bool pxw = x0 == 1 && pd[0] != kNoPush, pxe = x0 + 3 == nx && pd[1] != kNoPush;
  const bool pys = y == 1 && pd[2] != kNoPush, pyn = y == ny && pd[3] != kNoPush;
  auto ld4 = [](const float* p) { return *reinterpret_cast<const float4*>(p); };
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const long long row = (long long)y * sx + x0;
  // Rows y+-1 inside the block and off the walls make the mask of every cell
  // and neighbour a function of x alone (the fast path below; uniform across
  // a warp, which is one row when nx = 128).  Of the x positions x0-1 ..
  // x0+4 only x0 and x0+3 can be wall cells (nx is a multiple of 4) and only
  // x0-1 and x0+4 can lie outside the block (their zero-iterate value is 0).
  const bool fy = y >= 3 && y <= ny - 2;
  const float iv0 = ivtab[0];
  const float iv_0 = ivtab[x0 == 1 ? (ph & 1) : 0], iv_3 = ivtab[x0 + 3 == nx ? (ph & 2) : 0];
  const float ivw = x0 > 1 ? iv0 : 0.f, ive = x0 + 4 <= nx ? iv0 : 0.f;
  const float aw0 = (x0 == 1 && (ph & 1)) ? 0.f : ax, ae3 = (x0 + 3 == nx && (ph & 2)) ? 0.f : ax;
  // plane z of the own row and rows y+-1 and the cells beside the group, one
  // plane ahead of their use
  auto load_plane = [&](int z, float4& hs_, float4& hn_, float& rl_, float& rr_) {
    const long long o = (long long)z * sxy + row;
    hs_ = y > 1 ? ld4(R + o - sx) : zero4;
    hn_ = y < ny ? ld4(R + o + sx) : zero4;
    rl_ = x0 > 1 ? R[o - 1] : 0.f;
    rr_ = x0 + 4 <= nx ? R[o + 4] : 0.f;
  };
  float4 hb = zs > 1 ? ld4(R + (long long)(zs - 1) * sxy + row) : zero4;
  float4 hz = ld4(R + (long long)zs * sxy + row);
  float4 ht = zs < nz ? ld4(R + (long long)(zs + 1) * sxy + row) : zero4;
  float4 hs, hn;
  float rl, rr;
  load_plane(zs, hs, hn, rl, rr);
  for (int z = zs; z <= ze; ++z) {
    const long long o = (long long)z * sxy + row;
    float4 ht2 = zero4, hs2 = zero4, hn2 = zero4;
    float rl2 = 0.f, rr2 = 0.f;
    if (z < ze) {
      if (z + 1 < nz) ht2 = ld4(R + o + 2 * sxy);
      load_plane(z + 1, hs2, hn2, rl2, rr2);
    }
    const float hzv[4] = {hz.x, hz.y, hz.z, hz.w};
    const float hbv[4] = {hb.x, hb.y, hb.z, hb.w};
    const float htv[4] = {ht.x, ht.y, ht.z, ht.w};
    const float hsv[4] = {hs.x, hs.y, hs.z, hs.w};
    const float hnv[4] = {hn.x, hn.y, hn.z, hn.w};
    float out[4];
    const int par = (x0 + y + z) & 1;  // cell k is red when (x0 + k + y + z) is odd
    if (fy && z >= 3 && z <= nz - 2) {
      // the general update below with every mask a function of x: the same
      // products and the same fused chain
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float ivk = k == 0 ? iv_0 : (k == 3 ? iv_3 : iv0);
        if (((par + k) & 1) == 1) {
          out[k] = sorf(0.f, hzv[k] * ivk, om);
        } else {
          const float w = sorf(0.f, k > 0 ? hzv[k - 1] * (k == 1 ? iv_0 : iv0) : rl * ivw, om);
          const float e = sorf(0.f, k < 3 ? hzv[k + 1] * (k == 2 ? iv_3 : iv0) : rr * ive, om);
          const float aw = k == 0 ? aw0 : ax, ae = k == 3 ? ae3 : ax;
          const float sum = fmaf(az, sorf(0.f, htv[k] * ivk, om), fmaf(az, sorf(0.f, hbv[k] * ivk, om),
                            fmaf(ay, sorf(0.f, hnv[k] * ivk, om), fmaf(ay, sorf(0.f, hsv[k] * ivk, om),
                            fmaf(ae, e, aw * w)))));
          out[k] = sorf(0.f, (hzv[k] - sum) * ivk, om);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int x = x0 + k;
        const int m = wmask(x, y, z);
        const float iv = ivtab[m];
        if (((par + k) & 1) == 1) {
          out[k] = sorf(0.f, hzv[k] * iv, om);
        } else {
          // red neighbours (zero outside the block's interior)
          const float w = sorf(0.f, k > 0 ? hzv[k - 1] * ivtab[wmask(x - 1, y, z)] : (x0 > 1 ? rl * ivtab[wmask(x - 1, y, z)] : 0.f), om);
          const float e = sorf(0.f, k < 3 ? hzv[k + 1] * ivtab[wmask(x + 1, y, z)] : (x + 1 <= nx ? rr * ivtab[wmask(x + 1, y, z)] : 0.f), om);
          const float sv = sorf(0.f, y > 1 ? hsv[k] * ivtab[wmask(x, y - 1, z)] : 0.f, om);
          const float nv = sorf(0.f, y < ny ? hnv[k] * ivtab[wmask(x, y + 1, z)] : 0.f, om);
          const float bv = sorf(0.f, z > 1 ? hbv[k] * ivtab[wmask(x, y, z - 1)] : 0.f, om);
          const float tv = sorf(0.f, z < nz ? htv[k] * ivtab[wmask(x, y, z + 1)] : 0.f, om);
          const float aw = (m & 1) ? 0.f : ax, ae = (m & 2) ? 0.f : ax, as = (m & 4) ? 0.f : ay,
                      an = (m & 8) ? 0.f : ay, ab = (m & 16) ? 0.f : az, at = (m & 32) ? 0.f : az;
          const float sum = fmaf(at, tv, fmaf(ab, bv, fmaf(an, nv, fmaf(as, sv, fmaf(ae, e, aw * w)))));
          out[k] = sorf(0.f, (hzv[k] - sum) * iv, om);
        }
      }
    }
    const float4 v = make_float4(out[0], out[1], out[2], out[3]);
    float* q = D + o;
    *reinterpret_cast<float4*>(q) = v;
    if (pxw) q[pd[0]] = v.x;
    if (pxe) q[3 + pd[1]] = v.w;
    if (pys) *reinterpret_cast<float4*>(q + pd[2]) = v;
    if (pyn) *reinterpret_cast<float4*>(q + pd[3]) = v;
    if (z == 1 && pd[4] != kNoPush) *reinterpret_cast<float4*>(q + pd[4]) = v;
    if (z == nz && pd[5] != kNoPush) *reinterpret_cast<float4*>(q + pd[5]) = v;
    hb = hz;
    hz = ht;
    ht = ht2;
    hs = hs2;
    hn = hn2;
    rl = rl2;
    rr = rr2;
  }
}

}  // namespace

cudaError_t launch_rbgs_zero32(const BlkLev* bl, const Tile* tiles, int ntiles, int zc, const float* rhs, float* dst,
                               const long long* push, float om, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  pdl_launch(k_rbgs_zero32, ntiles, 256, 0, st, bl, tiles, zc, rhs, dst, push, om);
  return cudaGetLastError();
}

namespace {

// ---------------------------------------------------------------------------
// Sequential smoothers of mgrelax on the GPU: lexicographic Gauss-Seidel
// (mg_itrsch=1, mgsolver.for:407-432) and the line TDMA (mg_itrsch=2,
// :434-549).  Both are Gauss-Seidel orderings: the reference visits cells
// (lines) one after another and every cell (line) reads the already updated
// values of its predecessors.  On the GPU one CTA owns one block; cells
// (lines) whose predecessors are all done form a wavefront (a hyperplane
// x+y+z = const of cells, an anti-diagonal of lines) and are updated in
// parallel, with a CTA barrier between wavefronts, so every value is the
// one the sequential loop computes, with the reference's operand order.
// Blocks are independent within a sweep (their ghosts change only in the
// exchange after it), so blocks run as separate CTAs.  The sweep is out of
// place like the other smoothers: the CTA first copies its block, ghosts
// included, from src to dst (zeros for a zero iterate) and then works in
// place on dst.

// The block's cells, ghosts included, from src (or zeros) into dst.
template <typename T>
__device__ __forceinline__ void copy_block(const BlkLev& B, const T* __restrict__ S, T* __restrict__ D, bool zero) {
  const int ex = B.nx + 2, ey = B.ny + 2, ez = B.nz + 2;
  const long long n = (long long)ex * ey * ez;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const int x = (int)(q % ex), y = (int)((q / ex) % ey), z = (int)(q / ((long long)ex * ey));
    const long long i = (long long)z * B.sxy + (long long)y * B.sx + x;
    D[i] = zero ? T(0) : S[i];
  }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(512) k_gslex(const BlkLev* __restrict__ bls, const T* __restrict__ src,
                                               T* __restrict__ dst, const T* __restrict__ rhs,
                                               const T* __restrict__ fx, const T* __restrict__ fy,
                                               const T* __restrict__ fz, bool zero) {
  pdl_trigger();
  pdl_wait();
  const BlkLev B = bls[blockIdx.x];
  T* __restrict__ D = dst + B.off;
  const T* __restrict__ R = rhs + B.off;
  const T* FX = VAR ? fx + B.off : nullptr;
  const T* FY = VAR ? fy + B.off : nullptr;
  const T* FZ = VAR ? fz + B.off : nullptr;
  copy_block(B, src + B.off, D, zero);
  __syncthreads();
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sx = B.sx, sxy = B.sxy;
  // cell (x, y, z) is in wavefront d = (x-1) + (y-1) + (z-1)
  for (int d = 0; d <= (nx - 1) + (ny - 1) + (nz - 1); ++d) {
    const int zmin = max(0, d - (nx - 1) - (ny - 1)), zmax = min(nz - 1, d);
    const int nzr = zmax - zmin + 1;
    for (int q = threadIdx.x; q < nzr * ny; q += blockDim.x) {
      const int z = zmin + q / ny + 1, y = q % ny + 1;
      const int x = d - (y - 1) - (z - 1) + 1;
      if (x < 1 || x > nx) continue;
      const long long i = (long long)z * sxy + (long long)y * sx + x;
      const Coef<T> c = cell_coef<T, VAR>(B, x, y, z, i, FX, FY, FZ);
      D[i] = gs_div(R[i] - (c.aw * D[i - 1] + c.ae * D[i + 1] + c.as * D[i - sx] + c.an * D[i + sx] +
                            c.ab * D[i - sxy] + c.at * D[i + sxy]),
                    coef_ap(c));
    }
    __syncthreads();
  }
}

// One TDMA line of the block (AXIS 0: along x at (y, z) = (u, v); 1: along y
// at (x, z) = (u, v); 2: along z at (x, y) = (u, v)).  Forward elimination
// keeps the reference's recurrences, apr = 1/(ap - lo*a(s-1)), a(s) = hi*apr,
// c(s) = (su - <the four cross terms in the reference's order> - lo*c(s-1))*apr,
// with a(0) = 0 and c(0) the ghost before the line; back substitution
// phi(s) = c(s) - a(s)*phi(s+1) from the ghost after it.  c(s) is kept in the
// line's own cell (no other line of the wavefront reads it), a(s) in A.
template <typename T, bool VAR, int AXIS>
__device__ __forceinline__ void tdma_line(const BlkLev& B, T* __restrict__ D, T* __restrict__ A,
                                          const T* __restrict__ R, const T* FX, const T* FY, const T* FZ, int u,
                                          int v) {
  const long long sx = B.sx, sxy = B.sxy;
  const int n = AXIS == 0 ? B.nx : AXIS == 1 ? B.ny : B.nz;
  const long long st = AXIS == 0 ? 1 : AXIS == 1 ? sx : sxy;
  long long i = AXIS == 0 ? (long long)v * sxy + (long long)u * sx
                          : AXIS == 1 ? (long long)v * sxy + u : (long long)v * sx + u;  // position 0
  T aprev = T(0), cprev = D[i];
  for (int s = 1; s <= n; ++s) {
    i += st;
    const int x = AXIS == 0 ? s : u, y = AXIS == 0 ? u : AXIS == 1 ? s : v, z = AXIS == 2 ? s : v;
    const Coef<T> c = cell_coef<T, VAR>(B, x, y, z, i, FX, FY, FZ);
    const T ap = coef_ap(c);
    T lo, hi, t;
    if (AXIS == 1) {  // j-lines, mgsolver.for:443-473
      lo = c.as; hi = c.an;
      t = R[i] - c.ae * D[i + 1] - c.aw * D[i - 1] - c.at * D[i + sxy] - c.ab * D[i - sxy];
    } else if (AXIS == 0) {  // i-lines, :476-510
      lo = c.aw; hi = c.ae;
      t = R[i] - c.an * D[i + sx] - c.as * D[i - sx] - c.at * D[i + sxy] - c.ab * D[i - sxy];
    } else {  // k-lines, :513-547
      lo = c.ab; hi = c.at;
      t = R[i] - c.an * D[i + sx] - c.as * D[i - sx] - c.ae * D[i + 1] - c.aw * D[i - 1];
    }
    const T apr = gs_div(T(1), ap - lo * aprev);
    aprev = hi * apr;
    cprev = (t - lo * cprev) * apr;
    A[i] = aprev;
    D[i] = cprev;
  }
  T nxt = D[i + st];
  for (int s = n; s >= 1; --s) {
    nxt = D[i] - A[i] * nxt;
    D[i] = nxt;
    i -= st;
  }
}

// One pass of lines along AXIS: the reference runs them with the slower of
// the two other indices outer (j-lines: k then i; i-lines: k then j; k-lines:
// i then j), so line (u, v) follows (u-1, v) and (u, v-1): anti-diagonals
// u + v = const are the wavefronts.
template <typename T, bool VAR, int AXIS>
__device__ __forceinline__ void tdma_pass(const BlkLev& B, T* __restrict__ D, T* __restrict__ A,
                                          const T* __restrict__ R, const T* FX, const T* FY, const T* FZ) {
  const int nu = AXIS == 0 ? B.ny : B.nx, nv = AXIS == 2 ? B.ny : B.nz;
  for (int d = 0; d <= (nu - 1) + (nv - 1); ++d) {
    const int ulo = max(0, d - (nv - 1)), uhi = min(nu - 1, d);
    for (int u = ulo + (int)threadIdx.x; u <= uhi; u += blockDim.x)
      tdma_line<T, VAR, AXIS>(B, D, A, R, FX, FY, FZ, u + 1, d - u + 1);
    __syncthreads();
  }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_tdma(const BlkLev* __restrict__ bls, const T* __restrict__ src,
                                              T* __restrict__ dst, const T* __restrict__ rhs, T* __restrict__ acoef,
                                              const T* __restrict__ fx, const T* __restrict__ fy,
                                              const T* __restrict__ fz, bool zero) {
  pdl_trigger();
  pdl_wait();
  const BlkLev B = bls[blockIdx.x];
  T* __restrict__ D = dst + B.off;
  T* __restrict__ A = acoef + B.off;
  const T* __restrict__ R = rhs + B.off;
  const T* FX = VAR ? fx + B.off : nullptr;
  const T* FY = VAR ? fy + B.off : nullptr;
  const T* FZ = VAR ? fz + B.off : nullptr;
  copy_block(B, src + B.off, D, zero);
  __syncthreads();
  tdma_pass<T, VAR, 1>(B, D, A, R, FX, FY, FZ);  // j-lines
  tdma_pass<T, VAR, 0>(B, D, A, R, FX, FY, FZ);  // i-lines
  tdma_pass<T, VAR, 2>(B, D, A, R, FX, FY, FZ);  // k-lines
}

}  // namespace

template <typename T>
cudaError_t launch_seq_smoother(int itrsch, bool var, bool zero, const BlkLev* bl, int nb, const T* src, T* dst,
                                const T* rhs, T* acoef, const T* fx, const T* fy, const T* fz, cudaStream_t st) {
  if (nb <= 0) return cudaSuccess;
  if (itrsch == 1) {
    if (var) pdl_launch(k_gslex<T, true>, nb, 512, 0, st, bl, src, dst, rhs, fx, fy, fz, zero);
    else pdl_launch(k_gslex<T, false>, nb, 512, 0, st, bl, src, dst, rhs, fx, fy, fz, zero);
  } else {
    if (var) pdl_launch(k_tdma<T, true>, nb, 256, 0, st, bl, src, dst, rhs, acoef, fx, fy, fz, zero);
    else pdl_launch(k_tdma<T, false>, nb, 256, 0, st, bl, src, dst, rhs, acoef, fx, fy, fz, zero);
  }
  return cudaGetLastError();
}

template cudaError_t launch_seq_smoother<double>(int, bool, bool, const BlkLev*, int, const double*, double*,
                                                 const double*, double*, const double*, const double*,
                                                 const double*, cudaStream_t);
template cudaError_t launch_seq_smoother<float>(int, bool, bool, const BlkLev*, int, const float*, float*,
                                                const float*, float*, const float*, const float*, const float*,
                                                cudaStream_t);

namespace {


// Per-thread stencil state of the row-tile smoothers.  A thread's cells are
// fixed for the whole z march (pair k, member m: x = 2(tc + k*TPR) + 1 + m),
// so the constant coefficients of mgsolver.for:186-205 are selected once.
// FP64 keeps the reference's operand order and IEEE division (bit-exact);
// the FP32 inner solve uses fused multiply-adds and a reciprocal of the
// diagonal computed once per cell column.
template <typename T, int CP, bool VAR>
struct RowGs {
  T cw[CP][2], ce[CP][2], cinv[CP][2], cxy[CP][2];
  T cs, cn, az;
  float om;  // over-relaxation (FP32)
  int ph, nz;

  __device__ __forceinline__ void init(const BlkLev& B, int y, int tc, int tpr) {
    ph = B.phys;
    nz = B.nz;
    const T ax = (T)B.ax, ay = (T)B.ay;
    az = (T)B.az;
    cs = (y == 1 && (ph & 4)) ? T(0) : ay;
    cn = (y == B.ny && (ph & 8)) ? T(0) : ay;
#pragma unroll
    for (int k = 0; k < CP; ++k)
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int x = 2 * (tc + k * tpr) + 1 + m;
        cw[k][m] = (x == 1 && (ph & 1)) ? T(0) : ax;
        ce[k][m] = (x == B.nx && (ph & 2)) ? T(0) : ax;
        cxy[k][m] = cw[k][m] + ce[k][m] + cs + cn;
        cinv[k][m] = T(1) / (-(cxy[k][m] + az + az));
      }
  }

  // New value of the cell at smem index s (row pitch sp) of plane z, pair k,
  // member m; rv = its right-hand side; i = its offset in the block (VAR).
  __device__ __forceinline__ T update(const T* P, const T* Pm, const T* Pp, int s, int sp, int k, int m, int z,
                                      T rv, const T* FX, const T* FY, const T* FZ, long long i, int sx,
                                      long long sxy) const {
    T aw, ae, as, an, ab, at;
    if (VAR) {
      aw = FX[i - 1]; ae = FX[i]; as = FY[i - sx]; an = FY[i]; ab = FZ[i - sxy]; at = FZ[i];
    } else {
      aw = m ? cw[k][1] : cw[k][0];
      ae = m ? ce[k][1] : ce[k][0];
      as = cs;
      an = cn;
      ab = (z == 1 && (ph & 16)) ? T(0) : az;
      at = (z == nz && (ph & 32)) ? T(0) : az;
    }
    const T w = P[s - 1], e = P[s + 1], so = P[s - sp], no = P[s + sp], bo = Pm[s], to = Pp[s];
    if (sizeof(T) == 8) {
      const T ap = -(aw + ae + as + an + ab + at);
      return gs_div(rv - (aw * w + ae * e + as * so + an * no + ab * bo + at * to), ap);
    } else {
      const T sum = fma(at, to, fma(ab, bo, fma(an, no, fma(as, so, fma(ae, e, aw * w)))));
      T inv;
      if (!VAR && z > 1 && z < nz) inv = m ? cinv[k][1] : cinv[k][0];
      else inv = T(1) / (-(aw + ae + as + an + ab + at));
      return sorf(P[s], (rv - sum) * inv, om);
    }
  }
};

// ---------------------------------------------------------------------------
// Row-tile red-black sweep.  A CTA owns TY whole rows (x = 0..nx+1) of one
// block and marches a z range; because a tile spans the whole row there is no
// x halo, only one red halo row above and below.  Thread (tr, tc) owns the
// cell pairs p = tc + k*TPR (x = 2p+1, 2p+2) of row y0-1+tr: of every pair
// exactly one cell is red and one black, so neither colour phase diverges.
// Shared memory holds four staged planes of rows y0-2 .. y0+TY+1; column c
// holds x = c-1.  Same out-of-place contract and arithmetic as k_rbgs.
template <typename T, int TPR, int CP, int TY, bool VAR, bool ZERO>
__global__ void __launch_bounds__(TPR*(TY + 2)) k_rbgs_rows(const BlkLev* __restrict__ bls,
                                                           const Tile* __restrict__ tiles, int zc,
                                                           const T* __restrict__ src, T* __restrict__ dst,
                                                           const T* __restrict__ rhs, const T* __restrict__ fx,
                                                           const T* __restrict__ fy, const T* __restrict__ fz,
                                                           float om) {
  pdl_trigger();
  pdl_wait();
  constexpr int SP = 2 * CP * TPR + 4;
  constexpr int SR = TY + 4;
  constexpr int PL = SR * SP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sx = B.sx, sxy = B.sxy;
  const T* __restrict__ S = src + B.off;
  T* __restrict__ D = dst + B.off;
  const T* __restrict__ R = rhs + B.off;
  const T* FX = VAR ? fx + B.off : nullptr;
  const T* FY = VAR ? fy + B.off : nullptr;
  const T* FZ = VAR ? fz + B.off : nullptr;
  const int y0 = t.y0, zs = t.z0;
  const int ze = min(zs + zc - 1, nz);
  const int zlo = max(zs - 1, 1), zhi = min(ze + 1, nz);
  const int tr = threadIdx.x / TPR, tc = threadIdx.x - (threadIdx.x / TPR) * TPR;
  const int y = y0 - 1 + tr;
  const int srow = (tr + 1) * SP;
  const bool row_in = y >= 1 && y <= ny;
  const bool row_own = tr >= 1 && tr <= TY && y <= ny;
  const int ph = B.phys;
  const T ax = (T)B.ax, ay = (T)B.ay, az = (T)B.az;
  const T as_c = (y == 1 && (ph & 4)) ? T(0) : ay;
  const T an_c = (y == ny && (ph & 8)) ? T(0) : ay;

  auto stage = [&](int z) {
    T* P = ring + (z & 3) * PL;
    const T* Sz = S + (long long)z * sxy;
    for (int r = tr; r < SR; r += TY + 2) {
      const int yy = y0 - 2 + r;
      const bool yok = yy >= 0 && yy <= ny + 1;
      const T* Srow = Sz + (long long)yy * sx;
      T* Prow = P + r * SP + 1;
      for (int c = tc; c <= nx + 1; c += TPR) {
        T v = T(0);
        if (!ZERO && yok) v = Srow[c];
        Prow[c] = v;
      }
    }
  };
  // one cell update in plane z (P), neighbours in Pm (z-1), Pp (z+1)
  RowGs<T, CP, VAR> gs;
  gs.init(B, y, tc, TPR);
  gs.om = om;
  auto red = [&](int z) {
    if (!row_in) return;
    T* P = ring + (z & 3) * PL;
    const T* Pm = ring + ((z - 1) & 3) * PL;
    const T* Pp = ring + ((z + 1) & 3) * PL;
    const long long rowg = (long long)z * sxy + (long long)y * sx;
    const int j = (y + z) & 1;
#pragma unroll
    for (int k = 0; k < CP; ++k) {
      const int x = 2 * (tc + k * TPR) + 1 + j;
      if (x <= nx && H3D_IN(50, t.b, rowg + x, sxy * (nz + 2)) && H3D_IN(52, t.b, srow + x + 1 - SP, PL - 2 * SP))
        P[srow + x + 1] = gs.update(P, Pm, Pp, srow + x + 1, SP, k, j, z, R[rowg + x], FX, FY, FZ, rowg + x, (int)sx, sxy);
    }
  };
  auto black_store = [&](int z) {
    if (!row_own) return;
    T* P = ring + (z & 3) * PL;
    const T* Pm = ring + ((z - 1) & 3) * PL;
    const T* Pp = ring + ((z + 1) & 3) * PL;
    const long long rowg = (long long)z * sxy + (long long)y * sx;
    const int jb = (y + z + 1) & 1;
#pragma unroll
    for (int k = 0; k < CP; ++k) {
      const int xp = 2 * (tc + k * TPR) + 1;
      if (xp > nx) continue;
      const int xb = xp + jb, xr = xp + 1 - jb;
      if (!H3D_IN(51, t.b, rowg + xb, sxy * (nz + 2)) || !H3D_IN(53, t.b, srow + xb + 1 - SP, PL - 2 * SP)) continue;
      const T vr = P[srow + xr + 1];
      const T vb = gs.update(P, Pm, Pp, srow + xb + 1, SP, k, jb, z, R[rowg + xb], FX, FY, FZ, rowg + xb, (int)sx, sxy);
      D[rowg + xr] = vr;
      D[rowg + xb] = vb;
    }
  };

  stage(zlo - 1);
  stage(zlo);
  for (int z = zlo; z <= zhi; ++z) {
    stage(z + 1);
    __syncthreads();
    red(z);
    __syncthreads();
    if (z - 1 >= zs && z - 1 <= ze) black_store(z - 1);
    __syncthreads();
  }
  if (ze == nz) black_store(nz);
}


// ---------------------------------------------------------------------------
// Helpers of the TMA-staged sweeps: shared-memory addresses and bounded
// mbarrier waits.  No multicast is used anywhere.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// First 128-byte boundary of the dynamic shared memory, by pointer arithmetic
// on the shared array itself so that accesses through it stay shared-memory
// instructions (a round trip through an integer would make them generic).
__device__ __forceinline__ unsigned char* smem_base128(unsigned char* raw) {
  return raw + ((128u - (smem_u32(raw) & 127u)) & 127u);
}

// Bounded wait on an mbarrier phase: gives up after g_wait_clocks SM clocks
// (default 2^26, tens of ms; a plane copy takes microseconds; set at run time
// by set_wait_clocks), records the failure in *err and makes every later
// wait of this thread return at once, so a failed copy can never hang the
// kernel.  A thread whose wait gave up issues no further copies, and before
// its CTA exits the issuing thread waits (drain_ring, a fixed limit of its
// own) for the copies it already issued, so none lands after the CTA's shared
// memory is released.
__device__ long long g_wait_clocks = 1LL << 26;
constexpr long long kDrainClocks = 1LL << 31;

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ void mbar_wait(uint32_t bar, uint32_t parity, int* err, bool& bad) {
  if (bad || mbar_try(bar, parity)) return;
  const long long lim = g_wait_clocks;
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try(bar, parity)) return;
    if (clock64() - t0 > lim) {
      bad = true;
      atomicExch(err, 1);
      return;
    }
  }
}

// The copies of a ring whose planes first .. last went through slots
// q % ns (the (q - first) / ns -th use of the slot): waits for the last copy
// into every slot.
__device__ __forceinline__ void drain_ring(const uint64_t* bars, int ns, int first, int last, int* err) {
  for (int q = max(first, last - ns + 1); q <= last; ++q) {
    const uint32_t bar = smem_u32(bars + (unsigned)q % (unsigned)ns);
    const uint32_t parity = ((unsigned)(q - first) / (unsigned)ns) & 1u;
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
      if (clock64() - t0 > kDrainClocks) {
        atomicExch(err, 2);
        break;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Single-barrier TMA sweep (k_rbgs_tma2).
//
// Same cell mapping, arithmetic and out-of-place contract as k_rbgs_rows, but
// the global loads are off the z march:
//  * one elected thread brings each plane in by the Tensor Memory Accelerator:
//    a 3-D bulk tensor copy of the iterate (box = whole padded row width x
//    TY+4 rows from y0-2, rows outside the block read as zero) and one of the
//    right-hand side (rows y0-1 .. y0+TY) into a ring slot, both completing
//    on the slot's mbarrier, D planes ahead of the computation;
//  * the black update trails the red update by two planes, so one barrier
//    per plane suffices: phase z updates red cells of plane z (reading planes
//    z-1..z+1, writing plane z in shared memory) and black cells of plane
//    z-2 (reading only the red-updated planes z-3..z-1, writing global
//    memory).  The two never touch the same plane.
// Every wait is bounded; a wait that gives up sets *err and the sweep
// finishes without hanging (the host reports a timeout).
// A plane p is last read in phase p+3, so a ring of D+4 slots lets the copy
// of plane z+D+1 be issued right after the barrier that ends phase z.
template <typename T, int TPR, int CP, int TY, int D>
struct Tma2Cfg {
  static constexpr int NS = D + 4;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int SPMAX = ((2 * CP * TPR + 2 + kXOff + VEC - 1) / VEC) * VEC;
  static constexpr int PSLOT = ((SPMAX * (TY + 4) * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int RSLOT = ((SPMAX * (TY + 2) * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int SLOT = PSLOT + RSLOT;
  static constexpr size_t SMEM = (size_t)NS * SLOT + 128 + NS * 8;
};

template <typename T, int TPR, int CP, int TY, int D, bool VAR>
__global__ void __launch_bounds__(TPR*(TY + 2)) k_rbgs_tma2(const BlkLev* __restrict__ bls,
                                                           const Tile* __restrict__ tiles, int zc,
                                                           const CUtensorMap* __restrict__ maps,
                                                           const CUtensorMap* __restrict__ rmaps,
                                                           T* __restrict__ dst, const T* __restrict__ fx,
                                                           const T* __restrict__ fy, const T* __restrict__ fz,
                                                           int* err, float om) {
  pdl_trigger();
  pdl_wait();
  using C = Tma2Cfg<T, TPR, CP, TY, D>;
  constexpr int NS = C::NS;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_base128(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NS * C::SLOT);

  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const CUtensorMap* map = maps + t.b;
  const CUtensorMap* rmap = rmaps + t.b;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const int sx = B.sx;
  const long long sxy = B.sxy;
  T* __restrict__ Dst = dst + B.off;
  const T* FX = VAR ? fx + B.off : nullptr;
  const T* FY = VAR ? fy + B.off : nullptr;
  const T* FZ = VAR ? fz + B.off : nullptr;
  const int y0 = t.y0, zs = t.z0;
  const int ze = min(zs + zc - 1, nz);
  const int zlo = max(zs - 1, 1), zhi = min(ze + 1, nz);
  const int BX = ((nx + 2 + kXOff + C::VEC - 1) / C::VEC) * C::VEC;  // smem row pitch == TMA box width
  const uint32_t tx_bytes = (uint32_t)(BX * (2 * TY + 6) * (int)sizeof(T));
  const int tr = threadIdx.x / TPR, tc = threadIdx.x - (threadIdx.x / TPR) * TPR;
  const int y = y0 - 1 + tr;
  const int prow = (tr + 1) * BX + kXOff;  // cell (x, y) of an iterate slot (slot row 0 = y0-2)
  const int rrow = tr * BX + kXOff;        // cell (x, y) of a right-hand-side slot (slot row 0 = y0-1)
  const bool row_in = y >= 1 && y <= ny;
  const bool row_own = tr >= 1 && tr <= TY && y <= ny;
  const bool leader = threadIdx.x == 0;
  bool bad = false;

  if (leader) {
    for (int q = 0; q < NS; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + q)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  auto pslot = [&](int z) -> T* { return reinterpret_cast<T*>(base + (z % NS) * C::SLOT); };
  auto rslot = [&](int z) -> const T* { return reinterpret_cast<const T*>(base + (z % NS) * C::SLOT + C::PSLOT); };
  int last_q = -1;  // last plane issued (leader)
  auto issue = [&](int z) {  // leader only
    last_q = z;
    const uint32_t bar = smem_u32(bars + (z % NS));
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(pslot(z))),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y0 - 2), "r"(z), "r"(bar)
        : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(rslot(z))),
        "l"(reinterpret_cast<uint64_t>(rmap)), "r"(0), "r"(y0 - 1), "r"(z), "r"(bar)
        : "memory");
  };
  auto wait_plane = [&](int z) {
    const uint32_t parity = (uint32_t)(((z - zlo + 1) / NS) & 1);
    mbar_wait(smem_u32(bars + (z % NS)), parity, err, bad);
  };
  RowGs<T, CP, VAR> gs;
  gs.init(B, y, tc, TPR);
  gs.om = om;
  auto red = [&](int z) {
    if (!row_in) return;
    T* P = pslot(z);
    const T* Pm = pslot(z - 1);
    const T* Pp = pslot(z + 1);
    const T* Rr = rslot(z) + rrow;
    const int j = (y + z) & 1;
    const long long zo = (long long)z * sxy + (long long)y * sx;
#pragma unroll
    for (int k = 0; k < CP; ++k) {
      const int x = 2 * (tc + k * TPR) + 1 + j;
      if (x <= nx && H3D_IN(44, t.b, prow + x - BX, C::PSLOT / (int)sizeof(T) - 2 * BX))
        P[prow + x] = gs.update(P, Pm, Pp, prow + x, BX, k, j, z, Rr[x], FX, FY, FZ, zo + x, sx, sxy);
    }
  };
  auto black_store = [&](int z) {
    if (!row_own) return;
    const T* P = pslot(z);
    const T* Pm = pslot(z - 1);
    const T* Pp = pslot(z + 1);
    const T* Rr = rslot(z) + rrow;
    const long long zo = (long long)z * sxy + (long long)y * sx;
    T* Drow = Dst + zo;
    const int jb = (y + z + 1) & 1;
#pragma unroll
    for (int k = 0; k < CP; ++k) {
      const int xp = 2 * (tc + k * TPR) + 1;
      if (xp > nx) continue;
      const int xb = xp + jb, xr = xp + 1 - jb;
      if (!H3D_IN(45, t.b, zo + xb, sxy * (nz + 2)) || !H3D_IN(46, t.b, prow + xb - BX, C::PSLOT / (int)sizeof(T) - 2 * BX))
        continue;
      const T vr = P[prow + xr];
      const T vb = gs.update(P, Pm, Pp, prow + xb, BX, k, jb, z, Rr[xb], FX, FY, FZ, zo + xb, sx, sxy);
      Drow[xr] = vr;
      Drow[xb] = vb;
    }
  };

  if (leader)
    for (int q = zlo - 1; q <= min(zlo + D, zhi + 1); ++q) issue(q);
  wait_plane(zlo - 1);
  wait_plane(zlo);
  for (int z = zlo; z <= ze + 2; ++z) {
    if (z <= zhi) {
      wait_plane(z + 1);
      red(z);
    }
    if (z - 2 >= zs && z - 2 <= ze) black_store(z - 2);
    // this phase's shared-memory writes are ordered before the TMA that reuses their slot
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (leader && !bad && z + D + 1 <= zhi + 1) issue(z + D + 1);
  }
  if (leader && bad) drain_ring(bars, NS, zlo - 1, last_q, err);
}

// ---------------------------------------------------------------------------
// Vectorised single-barrier TMA sweep (k_rbgs_vec), FP32 with constant
// coefficients: the production smoother of the mixed solver's FP32 levels.
//
// Same phases as k_rbgs_tma2 (red of plane z and black of plane z-2 between
// two barriers, iterate and right-hand side staged by TMA into an NS-slot
// ring D planes ahead), but a thread owns GPT groups of four consecutive
// cells x0 .. x0+3 (x0 = 1 + 4g, g = j + k*TPR) of one row, two of each
// colour, and moves each group with 16-byte shared-memory loads and stores;
// the black phase writes the finished group to global memory as one 16-byte
// store (x0 is 16-byte aligned in the padded layout).  Only x0 can be a west
// wall cell and x0+3 an east wall cell (nx is a multiple of 4), so a group
// keeps two face coefficients and three diagonal reciprocals in registers.
// Needs nx a multiple of 4 and nx <= 4*TPR*GPT.
template <int TPR, int GPT, int TY, int NS, int D>
struct VecCfg {
  static constexpr int SPMAX = 4 * TPR * GPT + 8;  // >= roundup(nx + 2 + kXOff, 4)
  static constexpr int PSLOT = ((SPMAX * (TY + 4) * 4 + 127) / 128) * 128;
  static constexpr int RSLOT = ((SPMAX * (TY + 2) * 4 + 127) / 128) * 128;
  static constexpr int SLOT = PSLOT + RSLOT;
  static constexpr size_t SMEM = (size_t)NS * SLOT + 128 + NS * 8;
  static_assert(SMEM <= 232448, "ring exceeds shared memory");
};

template <int TPR, int GPT, int TY, int NS, int D>
__global__ void __launch_bounds__(TPR*(TY + 2)) k_rbgs_vec(const BlkLev* __restrict__ bls,
                                                          const Tile* __restrict__ tiles, int zc,
                                                          const CUtensorMap* __restrict__ maps,
                                                          const CUtensorMap* __restrict__ rmaps,
                                                          float* __restrict__ dst, int* err, float om) {
  pdl_trigger();
  pdl_wait();
  using C = VecCfg<TPR, GPT, TY, NS, D>;
  static_assert(D + 4 <= NS, "a plane is read until three phases after its own");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_base128(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NS * C::SLOT);

  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const CUtensorMap* map = maps + t.b;
  const CUtensorMap* rmap = rmaps + t.b;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sx = B.sx, sxy = B.sxy;
  const int y0 = t.y0, zs = t.z0;
  const int ze = min(zs + zc - 1, nz);
  const int zlo = max(zs - 1, 1), zhi = min(ze + 1, nz);
  const int BX = (nx + 2 + kXOff + 3) & ~3;  // smem row pitch == TMA box width
  const uint32_t tx_bytes = (uint32_t)(BX * (2 * TY + 6) * 4);
  const int tr = threadIdx.x / TPR, j = threadIdx.x % TPR;
  const int y = y0 - 1 + tr;
  const bool yin = y >= 1 && y <= ny;
  const bool yown = yin && tr >= 1 && tr <= TY;
  const int prow = (tr + 1) * BX + kXOff;  // cell (x, y) of an iterate slot sits at prow + x
  const int rrow = tr * BX + kXOff;        // ... of a right-hand-side slot at rrow + x
  float* __restrict__ Drow = dst + B.off + (long long)y * sx;
  const bool leader = threadIdx.x == 0;
  bool bad = false;

  // constant coefficients (mgsolver.for:186-205): walls zero the face term
  const int ph = B.phys;
  const float ax = (float)B.ax, ay = (float)B.ay, az = (float)B.az;
  const float as = (y == 1 && (ph & 4)) ? 0.f : ay;
  const float an = (y == ny && (ph & 8)) ? 0.f : ay;
  float aw0[GPT], ae3[GPT], inv0[GPT], inv3[GPT];
  const float inv12 = 1.f / (-(ax + ax + as + an + az + az));
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    const int x0 = 1 + 4 * (j + k * TPR);
    aw0[k] = (x0 == 1 && (ph & 1)) ? 0.f : ax;
    ae3[k] = (x0 + 3 == nx && (ph & 2)) ? 0.f : ax;
    inv0[k] = 1.f / (-(aw0[k] + ax + as + an + az + az));
    inv3[k] = 1.f / (-(ax + ae3[k] + as + an + az + az));
  }

  if (leader) {
    for (int q = 0; q < NS; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + q)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  auto slot_of = [&](int z) { return z % NS; };
  auto pslot = [&](int s) -> float* { return reinterpret_cast<float*>(base + s * C::SLOT); };
  auto rslot = [&](int s) -> const float* { return reinterpret_cast<const float*>(base + s * C::SLOT + C::PSLOT); };
  int last_q = -1;  // last plane issued (leader)
  auto issue = [&](int z) {  // leader only
    last_q = z;
    const int sl = slot_of(z);
    const uint32_t bar = smem_u32(bars + sl);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(pslot(sl))),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y0 - 2), "r"(z), "r"(bar)
        : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(rslot(sl))),
        "l"(reinterpret_cast<uint64_t>(rmap)), "r"(0), "r"(y0 - 1), "r"(z), "r"(bar)
        : "memory");
  };
  auto wait_plane = [&](int z) {
    const uint32_t parity = (uint32_t)(((z - zlo + 1) / NS) & 1);
    mbar_wait(smem_u32(bars + slot_of(z)), parity, err, bad);
  };
  auto upd = [](float w, float e, float s, float n, float b, float tt, float rv, float aw, float ae, float as_,
                float an_, float ab, float at, float iv) -> float {
    const float sum = fmaf(at, tt, fmaf(ab, b, fmaf(an_, n, fmaf(as_, s, fmaf(ae, e, aw * w)))));
    return (rv - sum) * iv;
  };
  // The inputs of one group update: the group, its row neighbours above and
  // below, the planes below and above, the right-hand side, and the cell left
  // (colour 0) or right (colour 1) of the group.
  struct In {
    float4 c, u, dn, bz, tz, rh;
    float side;
  };
  auto load = [&](In& in, int sp, int sm, int su, int x0, int q) {
    const float* P = pslot(sp);
    const int pc = prow + x0;
    in.c = *reinterpret_cast<const float4*>(P + pc);
    in.u = *reinterpret_cast<const float4*>(P + pc - BX);
    in.dn = *reinterpret_cast<const float4*>(P + pc + BX);
    in.bz = *reinterpret_cast<const float4*>(pslot(sm) + pc);
    in.tz = *reinterpret_cast<const float4*>(pslot(su) + pc);
    in.rh = *reinterpret_cast<const float4*>(rslot(sp) + rrow + x0);
    in.side = q == 0 ? P[pc - 1] : P[pc + 4];
  };
  // New values of the cells of colour q (positions q and q+2) of group k.
  auto compute = [&](In& in, int k, int z, int q) {
    const bool wlo = z == 1 && (ph & 16), whi = z == nz && (ph & 32);
    const float ab = wlo ? 0.f : az, at = whi ? 0.f : az;
    float i0 = inv0[k], i3 = inv3[k], i12 = inv12;
    if (wlo || whi) {  // wall plane: the diagonal changes
      i0 = 1.f / (-(aw0[k] + ax + as + an + ab + at));
      i3 = 1.f / (-(ax + ae3[k] + as + an + ab + at));
      i12 = 1.f / (-(ax + ax + as + an + ab + at));
    }
    float4& c = in.c;
    if (q == 0) {
      c.x = sorf(c.x, upd(in.side, c.y, in.u.x, in.dn.x, in.bz.x, in.tz.x, in.rh.x, aw0[k], ax, as, an, ab, at, i0), om);
      c.z = sorf(c.z, upd(c.y, c.w, in.u.z, in.dn.z, in.bz.z, in.tz.z, in.rh.z, ax, ax, as, an, ab, at, i12), om);
    } else {
      c.y = sorf(c.y, upd(c.x, c.z, in.u.y, in.dn.y, in.bz.y, in.tz.y, in.rh.y, ax, ax, as, an, ab, at, i12), om);
      c.w = sorf(c.w, upd(c.z, in.side, in.u.w, in.dn.w, in.bz.w, in.tz.w, in.rh.w, ax, ae3[k], as, an, ab, at, i3), om);
    }
  };

  if (leader)
    for (int q = zlo - 1; q <= min(zlo + D, zhi + 1); ++q) issue(q);
  wait_plane(zlo - 1);
  wait_plane(zlo);
  int s0 = slot_of(zlo);  // slot of plane z
  // ring slot of i in [-NS, 2 NS): a mask when the ring is a power of two
  auto wrap = [](int i) {
    if constexpr ((NS & (NS - 1)) == 0) return i & (NS - 1);
    else return i < 0 ? i + NS : (i >= NS ? i - NS : i);
  };
  for (int z = zlo; z <= ze + 2; ++z) {
    const bool red = z <= zhi && yin;                    // red cells of plane z
    const int zb = z - 2;
    const bool blk = zb >= zs && zb <= ze && yown;      // black cells of plane z-2
    if (z <= zhi) wait_plane(z + 1);
    const int qr = (y + z) & 1, qb = (y + zb + 1) & 1;
    const int sr = s0, sb = wrap(s0 - 2);
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      const int x0 = 1 + 4 * (j + k * TPR);
      if (x0 > nx) continue;
      // every load of the phase first, then the arithmetic, then the stores
      In ir, ib;
      if (red) load(ir, sr, wrap(sr - 1), wrap(sr + 1), x0, qr);
      if (blk) load(ib, sb, wrap(sb - 1), wrap(sb + 1), x0, qb);
      if (red) compute(ir, k, z, qr);
      if (blk) compute(ib, k, zb, qb);
      if (red) *reinterpret_cast<float4*>(pslot(sr) + prow + x0) = ir.c;
      if (blk) *reinterpret_cast<float4*>(Drow + (long long)zb * sxy + x0) = ib.c;
    }
    // this phase's shared-memory writes are ordered before the TMA that reuses their slot
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (leader && !bad && z + D + 1 <= zhi + 1) issue(z + D + 1);
    s0 = wrap(s0 + 1);
  }
  if (leader && bad) drain_ring(bars, NS, zlo - 1, last_q, err);
}

// ---------------------------------------------------------------------------
template <typename T, bool ZERO_OLD>
__global__ void k_fill(const uint32_t* __restrict__ dsts, const uint32_t* __restrict__ srcs, int64_t n,
                       T* __restrict__ out, const T* __restrict__ cur, const T* __restrict__ old) {
  pdl_trigger();
  // the gather tables are written once at setup: fetch the first entry
  // while the predecessor finishes
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s = 0, d = 0;
  if (e < n) {
    s = __ldg(srcs + e);
    d = __ldg(dsts + e);
  }
  pdl_wait();
  for (; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    T v;
    if (s & kOldFlag) v = ZERO_OLD ? T(0) : old[s & kIdxMask];
    else v = cur[s];
    out[d] = v;
    const int64_t en = e + (int64_t)gridDim.x * blockDim.x;
    if (en < n) {
      s = __ldg(srcs + en);
      d = __ldg(dsts + en);
    }
  }
}

// ---------------------------------------------------------------------------
// Row work: one warp per row (b, y, z) of a row table, grid-stride over rows.
// rows_start[b] is the first row of block b; a block has (ny+2)*(nz+2) rows
// (all rows) or ny*nz rows (interior rows).
struct RowRef {
  int b, y, z;
};
__device__ __forceinline__ RowRef row_of(const BlkLev* __restrict__ bls, const int* __restrict__ start, int nb,
                                         int rid, bool interior) {
  RowRef r;
  r.b = find_block(start, nb, rid);
  const int local = rid - __ldg(start + r.b);
  const BlkLev& B = bls[r.b];
  const int my = interior ? B.ny : B.ny + 2;
  r.z = local / my;
  r.y = local - r.z * my;
  if (interior) { r.y += 1; r.z += 1; }
  return r;
}

// mgrestr: resf = su - (A phi) on the fine interior (mgsolver.for:707-714),
// coarse rhs = 0.125 * sum of the 2x2x2 children, i fastest (:748-752).
template <typename T, bool VAR, bool ZERO>
__global__ void __launch_bounds__(256) k_restrict(const BlkLev* __restrict__ fine, const BlkLev* __restrict__ coarse,
                                                  const int* __restrict__ row_start, int nb, int nrows,
                                                  const T* __restrict__ phi, const T* __restrict__ rhs,
                                                  T* __restrict__ rhs_c, const T* __restrict__ fx,
                                                  const T* __restrict__ fy, const T* __restrict__ fz) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef rr = row_of(coarse, row_start, nb, rid, true);
    const BlkLev C = coarse[rr.b];
    const BlkLev F = fine[rr.b];
    const T* P = phi + F.off;
    const T* Rf = rhs + F.off;
    const T* FX = VAR ? fx + F.off : nullptr;
    const T* FY = VAR ? fy + F.off : nullptr;
    const T* FZ = VAR ? fz + F.off : nullptr;
    const int Y = rr.y, Z = rr.z;
    for (int X = 1 + lane; X <= C.nx; X += 32) {
      T sum = T(0);
#pragma unroll
      for (int dk = 0; dk < 2; ++dk)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
          for (int di = 0; di < 2; ++di) {
            const int x = 2 * X - 1 + di, y = 2 * Y - 1 + dj, z = 2 * Z - 1 + dk;
            const long long i = (long long)z * F.sxy + (long long)y * F.sx + x;
            T r;
            if (ZERO) {
              r = Rf[i] - T(0);
            } else {
              Coef<T> c = cell_coef<T, VAR>(F, x, y, z, i, FX, FY, FZ);
              const T ap = coef_ap(c);
              r = Rf[i] - (c.aw * P[i - 1] + c.ae * P[i + 1] + c.as * P[i - F.sx] + c.an * P[i + F.sx] +
                           c.ab * P[i - F.sxy] + c.at * P[i + F.sxy] + ap * P[i]);
            }
            sum = (di | dj | dk) ? sum + r : r;
          }
      rhs_c[C.off + (long long)Z * C.sxy + (long long)Y * C.sx + X] = T(0.125) * sum;
    }
  }
}

// ---------------------------------------------------------------------------
// mgcorr + mgbound: for every fine cell incl. ghosts, out = old[s] + P[s]/64
// where s is the cell's mgbound source (ghost coordinates on physical faces
// clamp to the adjacent interior, W,E,S,N,B,T composition) and P the
// trilinear (27,9,3,1) sum in the reference's term order (mgsolver.for:838-892).
template <typename T, bool ZERO_OLD>
__global__ void __launch_bounds__(256) k_prolong(const BlkLev* __restrict__ fine, const BlkLev* __restrict__ coarse,
                                                 const int* __restrict__ row_start, int nb, int nrows,
                                                 const T* __restrict__ phi_c, const T* __restrict__ old,
                                                 T* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef rr = row_of(fine, row_start, nb, rid, false);
    const BlkLev F = fine[rr.b];
    const BlkLev C = coarse[rr.b];
    const int ph = F.phys;
    const int y = rr.y, z = rr.z;
    int sy = y, sz = z;
    if (y == 0 && (ph & 4)) sy = 1;
    if (y == F.ny + 1 && (ph & 8)) sy = F.ny;
    if (z == 0 && (ph & 16)) sz = 1;
    if (z == F.nz + 1 && (ph & 32)) sz = F.nz;
    const int ly = sy >> 1, lz = sz >> 1;
    const T wy0 = (sy & 1) ? T(1) : T(3), wy1 = (sy & 1) ? T(3) : T(1);
    const T wz0 = (sz & 1) ? T(1) : T(3), wz1 = (sz & 1) ? T(3) : T(1);
    const T* Pc = phi_c + C.off + (long long)lz * C.sxy + (long long)ly * C.sx;
    const long long cy = C.sx, cz = C.sxy;
    const T* Orow = old + F.off + (long long)sz * F.sxy + (long long)sy * F.sx;
    T* Out = out + F.off + (long long)z * F.sxy + (long long)y * F.sx;
    for (int x = lane; x <= F.nx + 1; x += 32) {
      int sx = x;
      if (x == 0 && (ph & 1)) sx = 1;
      if (x == F.nx + 1 && (ph & 2)) sx = F.nx;
      const int lx = sx >> 1;
      const T wx0 = (sx & 1) ? T(1) : T(3), wx1 = (sx & 1) ? T(3) : T(1);
      const T* Q = Pc + lx;
      // term order (di,dj,dk): 000, 010, 001, 011, 100, 110, 101, 111
      T s = (wx0 * wy0 * wz0) * Q[0];
      s = s + (wx0 * wy1 * wz0) * Q[cy];
      s = s + (wx0 * wy0 * wz1) * Q[cz];
      s = s + (wx0 * wy1 * wz1) * Q[cy + cz];
      s = s + (wx1 * wy0 * wz0) * Q[1];
      s = s + (wx1 * wy1 * wz0) * Q[1 + cy];
      s = s + (wx1 * wy0 * wz1) * Q[1 + cz];
      s = s + (wx1 * wy1 * wz1) * Q[1 + cy + cz];
      const T o = ZERO_OLD ? T(0) : Orow[sx];
      Out[x] = o + s / T(64);
    }
  }
}

// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void block_reduce4(double a0, double a1, double a2, double a3, double* out) {
  __shared__ double sh[4][NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 = fmax(a2, __shfl_xor_sync(0xffffffffu, a2, o));
    a3 += __shfl_xor_sync(0xffffffffu, a3, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sh[0][w] = a0; sh[1][w] = a1; sh[2][w] = a2; sh[3][w] = a3; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int q = 0; q < NT / 32; ++q) { s0 += sh[0][q]; s1 += sh[1][q]; s2 = fmax(s2, sh[2][q]); s3 += sh[3][q]; }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
  }
}

// newsolv_mg.for:39-55 as defect correction: p += pp over the whole block
// (ghosts included, :40-48), then r = b - A p (mgrestr's residual form).
// One warp per level-1 row (all rows incl. ghosts); per-CTA partial sums.
template <typename TE, typename TR, bool HAS_E, bool VAR>
__global__ void __launch_bounds__(256) k_defect(const BlkLev* __restrict__ bls, const int* __restrict__ row_start,
                                                int nb, int nrows, const double* __restrict__ p,
                                                const TE* __restrict__ e, double* __restrict__ p_next,
                                                const double* __restrict__ bvec, TR* __restrict__ rhs_out,
                                                double mean_b, double rscale, const double* __restrict__ fx,
                                                const double* __restrict__ fy, const double* __restrict__ fz,
                                                double* __restrict__ partials) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  double rr = 0, bb = 0, rm = 0, rs = 0;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef ref = row_of(bls, row_start, nb, rid, false);
    const BlkLev B = bls[ref.b];
    const int y = ref.y, z = ref.z;
    const bool row_in = y >= 1 && y <= B.ny && z >= 1 && z <= B.nz;
    const long long rowg = B.off + (long long)z * B.sxy + (long long)y * B.sx;
    auto pv = [&](long long j) -> double {
      if (HAS_E) return p[j] + (double)e[j];
      return p[j];
    };
    for (int x = lane; x <= B.nx + 1; x += 32) {
      const long long i = rowg + x;
      const double pc = pv(i);
      if (HAS_E) p_next[i] = pc;
      if (row_in && x >= 1 && x <= B.nx) {
        Coef<double> c = cell_coef<double, VAR>(B, x, y, z, i - B.off, VAR ? fx + B.off : nullptr,
                                                VAR ? fy + B.off : nullptr, VAR ? fz + B.off : nullptr);
        const double ap = coef_ap(c);
        const double bv = bvec[i];
        const double r = bv - (c.aw * pv(i - 1) + c.ae * pv(i + 1) + c.as * pv(i - B.sx) + c.an * pv(i + B.sx) +
                               c.ab * pv(i - B.sxy) + c.at * pv(i + B.sxy) + ap * pc);
        rhs_out[i] = (TR)(r - mean_b);
        rr += r * r;
        bb += bv * bv;
        rm = fmax(rm, fabs(r) * (rscale < 0.0 ? B.dv : rscale));
        rs += r;
      }
    }
  }
  block_reduce4<256>(rr, bb, rm, rs, partials + 4 * (size_t)blockIdx.x);
}


// ---------------------------------------------------------------------------
// Tile restriction (mgrestr, mgsolver.for:693-756).  A CTA owns TYC coarse
// rows x all coarse x of one block and marches the fine planes of a coarse z
// range, staging fine iterate planes (rows 2Y0-2 .. 2Y0+2TYC-1) in a 3-plane
// ring.  Each thread keeps the running sum of its coarse cells and adds the
// eight child residuals in the reference order (i fastest, then j, then k).
template <typename T, bool VAR, bool ZERO, int TPR, int CPX, int TYC>
__global__ void __launch_bounds__(TPR* TYC) k_restrict_tile(const BlkLev* __restrict__ fine,
                                                           const BlkLev* __restrict__ coarse,
                                                           const Tile* __restrict__ tiles, int zc,
                                                           const T* __restrict__ phi, const T* __restrict__ rhs,
                                                           T* __restrict__ rhs_c, const T* __restrict__ fx,
                                                           const T* __restrict__ fy, const T* __restrict__ fz) {
  pdl_trigger();
  pdl_wait();
  constexpr int SP = 2 * CPX * TPR + 4;
  constexpr int SR = 2 * TYC + 2;
  constexpr int PL = SR * SP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  const Tile t = tiles[blockIdx.x];
  const BlkLev F = fine[t.b];
  const BlkLev C = coarse[t.b];
  const T* P = phi + F.off;
  const T* Rf = rhs + F.off;
  const T* FX = VAR ? fx + F.off : nullptr;
  const T* FY = VAR ? fy + F.off : nullptr;
  const T* FZ = VAR ? fz + F.off : nullptr;
  const int Y0 = t.y0, Z0 = t.z0;
  const int Z1 = min(Z0 + zc - 1, C.nz);
  const int tr = threadIdx.x / TPR, tc = threadIdx.x - (threadIdx.x / TPR) * TPR;
  const int Y = Y0 + tr;
  const int fy0 = 2 * Y0 - 2;  // fine row held in smem row 0
  auto stage = [&](int zf) {
    T* S = ring + (zf % 3) * PL;
    const T* Pz = P + (long long)zf * F.sxy;
    for (int r = tr; r < SR; r += TYC) {
      const int yy = fy0 + r;
      if (yy < 0 || yy > F.ny + 1) continue;
      const T* row = Pz + (long long)yy * F.sx;
      T* srow = S + r * SP;
      for (int x = tc; x <= F.nx + 1; x += TPR)
        if (H3D_IN(10, t.b, (S - ring) + r * SP + x, 3 * PL) &&
            H3D_IN(11, t.b, (long long)zf * F.sxy + (long long)yy * F.sx + x, F.sxy * (F.nz + 2)))
          srow[x] = ZERO ? T(0) : row[x];
    }
  };
  T sum[CPX];
#pragma unroll
  for (int k = 0; k < CPX; ++k) sum[k] = T(0);
  stage(2 * Z0 - 2);
  stage(2 * Z0 - 1);
  for (int zf = 2 * Z0 - 1; zf <= 2 * Z1; ++zf) {
    stage(zf + 1);
    __syncthreads();
    if (Y <= C.ny) {
      const T* S = ring + (zf % 3) * PL;
      const T* Sm = ring + ((zf - 1) % 3) * PL;
      const T* Sp = ring + ((zf + 1) % 3) * PL;
#pragma unroll
      for (int k = 0; k < CPX; ++k) {
        const int X = 1 + tc + k * TPR;
        if (X > C.nx) continue;
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
          for (int di = 0; di < 2; ++di) {
            const int x = 2 * X - 1 + di, y = 2 * Y - 1 + dj;
            const long long i = (long long)zf * F.sxy + (long long)y * F.sx + x;
            T r = T(0);
            if (!H3D_IN(12, t.b, i, F.sxy * (F.nz + 2))) {
            } else if (ZERO) {
              r = Rf[i] - T(0);
            } else if (!H3D_IN(13, t.b, (y - fy0) * SP + x - SP, PL - 2 * SP)) {
            } else {
              const int q = (y - fy0) * SP + x;
              Coef<T> c = cell_coef<T, VAR>(F, x, y, zf, i, FX, FY, FZ);
              const T ap = coef_ap(c);
              r = Rf[i] - (c.aw * S[q - 1] + c.ae * S[q + 1] + c.as * S[q - SP] + c.an * S[q + SP] +
                           c.ab * Sm[q] + c.at * Sp[q] + ap * S[q]);
            }
            sum[k] = ((zf & 1) && dj == 0 && di == 0) ? r : sum[k] + r;
          }
        if (!(zf & 1) && H3D_IN(14, t.b, (long long)(zf >> 1) * C.sxy + (long long)Y * C.sx + X, C.sxy * (C.nz + 2)))
          rhs_c[C.off + (long long)(zf >> 1) * C.sxy + (long long)Y * C.sx + X] = T(0.125) * sum[k];
      }
    }
    __syncthreads();
  }
}

// mgcorr + mgbound with one thread per fine cell pair (2q, 2q+1) of a row:
// both cells of a pair interpolate from the same eight coarse cells.
template <typename T, bool ZERO_OLD>
__global__ void __launch_bounds__(256) k_prolong_pairs(const BlkLev* __restrict__ fine,
                                                       const BlkLev* __restrict__ coarse,
                                                       const int* __restrict__ row_start, int nb, int nrows,
                                                       const T* __restrict__ phi_c, const T* __restrict__ old,
                                                       T* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef rr = row_of(fine, row_start, nb, rid, false);
    const BlkLev F = fine[rr.b];
    const BlkLev C = coarse[rr.b];
    const int ph = F.phys;
    const int y = rr.y, z = rr.z;
    int sy = y, sz = z;
    if (y == 0 && (ph & 4)) sy = 1;
    if (y == F.ny + 1 && (ph & 8)) sy = F.ny;
    if (z == 0 && (ph & 16)) sz = 1;
    if (z == F.nz + 1 && (ph & 32)) sz = F.nz;
    const T wy0 = (sy & 1) ? T(1) : T(3), wy1 = (sy & 1) ? T(3) : T(1);
    const T wz0 = (sz & 1) ? T(1) : T(3), wz1 = (sz & 1) ? T(3) : T(1);
    const T w00 = wy0 * wz0, w10 = wy1 * wz0, w01 = wy0 * wz1, w11 = wy1 * wz1;  // [dj][dk]
    const T* Pc = phi_c + C.off + (long long)(sz >> 1) * C.sxy + (long long)(sy >> 1) * C.sx;
    const long long cy = C.sx, cz = C.sxy;
    const T* Orow = old + F.off + (long long)sz * F.sxy + (long long)sy * F.sx;
    T* Out = out + F.off + (long long)z * F.sxy + (long long)y * F.sx;
    const int npairs = (F.nx + 2) >> 1;
    for (int q = lane; q < npairs; q += 32) {
      const T* Q = Pc + q;
      if (!H3D_IN(20, rr.b, (long long)(sz >> 1) * C.sxy + (long long)(sy >> 1) * C.sx + q + 1 + cy + cz,
                  C.sxy * (C.nz + 2)))
        continue;
      const T c000 = Q[0], c010 = Q[cy], c001 = Q[cz], c011 = Q[cy + cz];
      const T c100 = Q[1], c110 = Q[1 + cy], c101 = Q[1 + cz], c111 = Q[1 + cy + cz];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int x = 2 * q + m;
        int sx = x;
        if (x == 0 && (ph & 1)) sx = 1;
        if (x == F.nx + 1 && (ph & 2)) sx = F.nx;
        const T wx0 = (sx & 1) ? T(1) : T(3), wx1 = (sx & 1) ? T(3) : T(1);
        // term order (di,dj,dk): 000, 010, 001, 011, 100, 110, 101, 111 (mgsolver.for:838-892)
        T s = (wx0 * w00) * c000;
        s = s + (wx0 * w10) * c010;
        s = s + (wx0 * w01) * c001;
        s = s + (wx0 * w11) * c011;
        s = s + (wx1 * w00) * c100;
        s = s + (wx1 * w10) * c110;
        s = s + (wx1 * w01) * c101;
        s = s + (wx1 * w11) * c111;
        if (!H3D_IN(21, rr.b, (long long)sz * F.sxy + (long long)sy * F.sx + sx, F.sxy * (F.nz + 2)) ||
            !H3D_IN(22, rr.b, (long long)z * F.sxy + (long long)y * F.sx + x, F.sxy * (F.nz + 2)))
          continue;
        const T o = ZERO_OLD ? T(0) : Orow[sx];
        Out[x] = o + s / T(64);
      }
    }
  }
}

__global__ void __launch_bounds__(1024) k_reduce4(const double* __restrict__ partials, int n, double* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (int q = threadIdx.x; q < n; q += 1024) {
    a0 += partials[4 * (size_t)q];
    a1 += partials[4 * (size_t)q + 1];
    a2 = fmax(a2, partials[4 * (size_t)q + 2]);
    a3 += partials[4 * (size_t)q + 3];
  }
  block_reduce4<1024>(a0, a1, a2, a3, out);
}

// Per-block sums of the defect partials: CTA b reduces partials
// start[b] .. start[b+1]-1 (the tiles of block b) in a fixed order.
__global__ void __launch_bounds__(256) k_reduce4_blocks(const double* __restrict__ partials,
                                                        const int* __restrict__ start, double* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const int b = blockIdx.x;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (int q = start[b] + threadIdx.x; q < start[b + 1]; q += 256) {
    a0 += partials[4 * (size_t)q];
    a1 += partials[4 * (size_t)q + 1];
    a2 = fmax(a2, partials[4 * (size_t)q + 2]);
    a3 += partials[4 * (size_t)q + 3];
  }
  block_reduce4<256>(a0, a1, a2, a3, out + 4 * (size_t)b);
}

// Sum of a field over the interior cells: a warp a row at a time (grid-stride
// over the level's interior rows), one partial sum per CTA in a fixed order.
__global__ void __launch_bounds__(256) k_sum_interior(const BlkLev* __restrict__ bls, const int* __restrict__ row_start,
                                                      int nb, int nrows, const double* __restrict__ a,
                                                      double* __restrict__ partials) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  double s = 0;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef rr = row_of(bls, row_start, nb, rid, true);
    const BlkLev& B = bls[rr.b];
    const double* row = a + B.off + (long long)rr.z * B.sxy + (long long)rr.y * B.sx;
    for (int x = 1 + lane; x <= B.nx; x += 32) s += row[x];
  }
  block_reduce4<256>(s, 0.0, 0.0, 0.0, partials + 4 * (size_t)blockIdx.x);
}

__global__ void k_shift(double* __restrict__ a, int64_t n, const double* __restrict__ s, double scale) {
  pdl_trigger();
  pdl_wait();
  const double v = s[0] * scale;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    a[q] = a[q] - v;
}

__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  pdl_trigger();
  pdl_wait();
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    b[q] = (float)a[q];
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
  pdl_trigger();
  pdl_wait();
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    b[q] = (double)a[q];
}

// dens_mg of level g = 0.125 * sum of the 8 children of level g-1 in the
// order of mgsolver.for:91-104 (j fastest, then i, then k).
__global__ void __launch_bounds__(256) k_dens_restrict(const BlkLev* __restrict__ fine, const BlkLev* __restrict__ coarse,
                                                       const int* __restrict__ cta_start, int nb,
                                                       const double* __restrict__ df, double* __restrict__ dc) {
  pdl_trigger();
  pdl_wait();
  const int b = find_block(cta_start, nb, blockIdx.x);
  const BlkLev C = coarse[b], F = fine[b];
  const int local = (blockIdx.x - cta_start[b]) * blockDim.x + threadIdx.x;
  if (local >= C.nx * C.ny * C.nz) return;
  const int X = local % C.nx + 1, Y = (local / C.nx) % C.ny + 1, Z = local / (C.nx * C.ny) + 1;
  const double* P = df + F.off + (long long)(2 * Z - 1) * F.sxy + (long long)(2 * Y - 1) * F.sx + (2 * X - 1);
  const long long I = 1, J = F.sx, K = F.sxy;
  double s = P[0] + P[J] + P[I] + P[I + J] + P[K] + P[K + J] + P[K + I] + P[K + I + J];
  dc[C.off + (long long)Z * C.sxy + (long long)Y * C.sx + X] = 0.125 * s;
}

// L_LSM face coefficients (mgsolver.for:130-184): face arrays at the cell
// index of the lower cell; block faces use the cell's own density; the
// fine-level dx, dy, dz are used at every level; physical faces are zeroed
// (:194-205).
__global__ void __launch_bounds__(256) k_face_coef(const BlkLev* __restrict__ bls, const int* __restrict__ cta_start,
                                                   int nb, const double* __restrict__ dens,
                                                   const double* __restrict__ h3, double* __restrict__ fx,
                                                   double* __restrict__ fy, double* __restrict__ fz) {
  pdl_trigger();
  pdl_wait();
  const int b = find_block(cta_start, nb, blockIdx.x);
  const BlkLev B = bls[b];
  const int local = (blockIdx.x - cta_start[b]) * blockDim.x + threadIdx.x;
  const int mx = B.nx + 2, my = B.ny + 2, mz = B.nz + 2;
  if (local >= mx * my * mz) return;
  const int x = local % mx, y = (local / mx) % my, z = local / (mx * my);
  const double dx = h3[3 * b], dy = h3[3 * b + 1], dz = h3[3 * b + 2];
  const long long i = B.off + (long long)z * B.sxy + (long long)y * B.sx + x;
  const bool iny = y >= 1 && y <= B.ny, inz = z >= 1 && z <= B.nz, inx = x >= 1 && x <= B.nx;
  // x faces: x in [0, nx]
  if (x <= B.nx && iny && inz) {
    double d;
    if (x == 0) d = dens[i + 1];
    else if (x == B.nx) d = dens[i];
    else d = 0.5 * (dens[i] + dens[i + 1]);
    double v = dy * dz / dx / d;
    if ((x == 0 && (B.phys & 1)) || (x == B.nx && (B.phys & 2))) v = 0.0;
    fx[i] = v;
  }
  if (y <= B.ny && inx && inz) {
    double d;
    if (y == 0) d = dens[i + B.sx];
    else if (y == B.ny) d = dens[i];
    else d = 0.5 * (dens[i] + dens[i + B.sx]);
    double v = dx * dz / dy / d;
    if ((y == 0 && (B.phys & 4)) || (y == B.ny && (B.phys & 8))) v = 0.0;
    fy[i] = v;
  }
  if (z <= B.nz && inx && iny) {
    double d;
    if (z == 0) d = dens[i + B.sxy];
    else if (z == B.nz) d = dens[i];
    else d = 0.5 * (dens[i] + dens[i + B.sxy]);
    double v = dx * dy / dz / d;
    if ((z == 0 && (B.phys & 16)) || (z == B.nz && (B.phys & 32))) v = 0.0;
    fz[i] = v;
  }
}

inline int grid_for(int64_t n, int nt) {
  int64_t g = (n + nt - 1) / nt;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

// ---------------------------------------------------------------------------
// Smoother variants: 0-7 generic tiles (k_rbgs), 8+ row tiles (k_rbgs_rows,
// tx = largest supported nx).
static const TileShape kShapes[] = {
    {32, 16, 256, false, 0, 0, 0, -1}, {32, 8, 256, false, 0, 0, 0, -1},
    {64, 8, 256, false, 0, 0, 0, -1},  {16, 8, 128, false, 0, 0, 0, -1},
    {8, 8, 64, false, 0, 0, 0, -1},    {8, 4, 32, false, 0, 0, 0, -1},
    {4, 4, 32, false, 0, 0, 0, -1},    {64, 16, 512, false, 0, 0, 0, -1},
    {128, 8, 640, true, 64, 1, 0, -1}, {128, 8, 320, true, 32, 2, 0, -1},   // 8, 9
    {64, 8, 320, true, 32, 1, 0, -1},  {64, 16, 576, true, 32, 1, 0, -1},   // 10, 11
    {32, 16, 288, true, 16, 1, 0, -1}, {16, 16, 144, true, 8, 1, 0, -1},    // 12, 13
    {256, 8, 640, true, 64, 2, 0, -1}, {128, 4, 384, true, 64, 1, 0, -1},   // 14, 15
    {256, 4, 768, true, 128, 1, 0, -1}, {128, 4, 192, true, 32, 2, 0, -1},  // 16, 17
    {256, 8, 320, true, 32, 4, 0, -1},                                          // 18
    {128, 4, 192, true, 32, 2, 2, 17},  {128, 8, 320, true, 32, 2, 2, 9},           // 19, 20
    {128, 4, 384, true, 64, 1, 2, 15},  {128, 8, 640, true, 64, 1, 2, 8},           // 21, 22
    {64, 8, 320, true, 32, 1, 2, 10},   {64, 16, 576, true, 32, 1, 2, 11},          // 23, 24
    {32, 16, 288, true, 16, 1, 2, 12},  {128, 16, 576, true, 32, 2, 2, 29},         // 25, 26
    {128, 8, 320, true, 32, 2, 2, 9},   {16, 16, 144, true, 8, 1, 2, 13},           // 27, 28
    {128, 16, 576, true, 32, 2, 0, -1},                                             // 29
    // vectorised FP32 sweeps (k_rbgs_vec); tpr = threads per row, cp = groups of four cells per thread
    {128, 4, 192, true, 32, 1, 3, 17},  {128, 8, 320, true, 32, 1, 3, 9},           // 30, 31
    {128, 8, 320, true, 32, 1, 3, 9},   {128, 16, 576, true, 32, 1, 3, 29},         // 32, 33
    {128, 8, 160, true, 16, 2, 3, 9},   {128, 16, 288, true, 16, 2, 3, 29},         // 34, 35
    {64, 8, 160, true, 16, 1, 3, 10},   {64, 16, 288, true, 16, 1, 3, 11},          // 36, 37
    {32, 16, 144, true, 8, 1, 3, 12},   {16, 16, 72, true, 4, 1, 3, 13},            // 38, 39
    // register-window FP32 sweeps (k_rbgs_win); tpr = lanes per row, one group each
    {128, 4, 192, true, 32, 1, 3, 17},  {128, 8, 320, true, 32, 1, 3, 9},           // 40, 41
    {128, 16, 576, true, 32, 1, 3, 29}, {128, 8, 320, true, 32, 1, 3, 9},           // 42, 43
    {64, 8, 160, true, 16, 1, 3, 10},   {64, 16, 288, true, 16, 1, 3, 11},          // 44, 45
    {32, 16, 144, true, 8, 1, 3, 12},   {16, 16, 72, true, 4, 1, 3, 13},            // 46, 47
    // register-window sweeps with two groups per lane
    {128, 16, 288, true, 16, 2, 3, 29}, {128, 8, 160, true, 16, 2, 3, 9},           // 48, 49
    {64, 16, 144, true, 8, 2, 3, 11},                                               // 50
    // register-window sweeps with the z march unrolled over the window
    {128, 8, 320, true, 32, 1, 3, 9},   {128, 16, 576, true, 32, 1, 3, 29},         // 51, 52
    {128, 8, 320, true, 32, 1, 3, 9},   {64, 8, 160, true, 16, 1, 3, 10},           // 53, 54
    {64, 16, 288, true, 16, 1, 3, 11},  {32, 16, 144, true, 8, 1, 3, 12},           // 55, 56
    {128, 8, 160, true, 16, 2, 3, 9},   {128, 4, 192, true, 32, 1, 3, 17},          // 57, 58
    // 15-row tiles: nine a 128-row block, so 16 such blocks give 144 CTAs, one per SM on 148 SMs
    {128, 15, 544, true, 32, 1, 3, -1}, {128, 15, 544, true, 32, 1, 3, -1},         // 59, 60
};
#ifdef H3D_BOUNDS_CHECK
// Debug builds only: first recorded out-of-bounds access {kernel id + 1, block, index, limit}.
extern "C" int h3d_debug_bounds(unsigned long long* out) {
  if (cudaMemcpyFromSymbol(out, g_h3d_bad, 4 * sizeof(unsigned long long)) != cudaSuccess) return -2;
  return 0;
}
#endif
int tma_ty_index(int ty) { return ty == 4 ? 0 : ty == 8 ? 1 : ty == 16 ? 2 : ty == 32 ? 3 : ty == 15 ? 4 : -1; }
int num_tile_shapes() { return (int)(sizeof(kShapes) / sizeof(kShapes[0])); }
TileShape tile_shape(int v) { return kShapes[v]; }

template <typename T, int TX, int TY, int NT>
static cudaError_t rbgs_dispatch(bool var, bool zero, const BlkLev* bl, const Tile* tiles, int ntiles, int zc,
                                 const T* src, T* dst, const T* rhs, const T* fx, const T* fy, const T* fz,
                                 float om, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  dim3 grid(ntiles), block(NT);
  if (var) {
    if (zero) pdl_launch(k_rbgs<T, TX, TY, NT, true, true>, grid, block, 0, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
    else pdl_launch(k_rbgs<T, TX, TY, NT, true, false>, grid, block, 0, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
  } else {
    if (zero) pdl_launch(k_rbgs<T, TX, TY, NT, false, true>, grid, block, 0, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
    else pdl_launch(k_rbgs<T, TX, TY, NT, false, false>, grid, block, 0, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
  }
  return cudaGetLastError();
}

template <typename T, int TPR, int CP, int TY>
static constexpr size_t rows_smem() {
  return 4 * (size_t)(TY + 4) * (size_t)(2 * CP * TPR + 4) * sizeof(T);
}

template <typename T, int TPR, int CP, int TY>
static cudaError_t rows_attr() {
  const int sm = (int)rows_smem<T, TPR, CP, TY>();
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_rbgs_rows<T, TPR, CP, TY, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  if ((e = cudaFuncSetAttribute(k_rbgs_rows<T, TPR, CP, TY, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  if ((e = cudaFuncSetAttribute(k_rbgs_rows<T, TPR, CP, TY, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  return cudaFuncSetAttribute(k_rbgs_rows<T, TPR, CP, TY, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

template <typename T, int TPR, int CP, int TY>
static cudaError_t rows_dispatch(bool var, bool zero, const BlkLev* bl, const Tile* tiles, int ntiles, int zc,
                                 const T* src, T* dst, const T* rhs, const T* fx, const T* fy, const T* fz,
                                 float om, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  constexpr int NT = TPR * (TY + 2);
  constexpr size_t SM = rows_smem<T, TPR, CP, TY>();
  dim3 grid(ntiles), block(NT);
  if (var) {
    if (zero) pdl_launch(k_rbgs_rows<T, TPR, CP, TY, true, true>, grid, block, SM, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
    else pdl_launch(k_rbgs_rows<T, TPR, CP, TY, true, false>, grid, block, SM, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
  } else {
    if (zero) pdl_launch(k_rbgs_rows<T, TPR, CP, TY, false, true>, grid, block, SM, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
    else pdl_launch(k_rbgs_rows<T, TPR, CP, TY, false, false>, grid, block, SM, st, bl, tiles, zc, src, dst, rhs, fx, fy, fz, om);
  }
  return cudaGetLastError();
}


// Prefetch depth actually used: the requested D, lowered until the ring fits
// in the 227 KB of shared memory a CTA may have.
template <typename T, int TPR, int CP, int TY, int D>
constexpr int tma2_depth() {
  if constexpr (D <= 1 || Tma2Cfg<T, TPR, CP, TY, D>::SMEM <= 232448) return D;
  else return tma2_depth<T, TPR, CP, TY, D - 1>();
}

template <typename T, int TPR, int CP, int TY, int D0>
static cudaError_t tma2_attr() {
  constexpr int D = tma2_depth<T, TPR, CP, TY, D0>();
  static_assert(Tma2Cfg<T, TPR, CP, TY, D>::SMEM <= 232448, "TMA ring exceeds shared memory");
  const int sm = (int)Tma2Cfg<T, TPR, CP, TY, D>::SMEM;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_rbgs_tma2<T, TPR, CP, TY, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  return cudaFuncSetAttribute(k_rbgs_tma2<T, TPR, CP, TY, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

template <typename T, int TPR, int CP, int TY, int D0>
static cudaError_t tma2_dispatch(bool var, const BlkLev* bl, const Tile* tiles, int ntiles, int zc,
                                 const CUtensorMap* maps, const CUtensorMap* rmaps, int* err, T* dst, const T* fx,
                                 const T* fy, const T* fz, float om, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  constexpr int D = tma2_depth<T, TPR, CP, TY, D0>();
  constexpr int NT = TPR * (TY + 2);
  constexpr size_t SM = Tma2Cfg<T, TPR, CP, TY, D>::SMEM;
  if (var) pdl_launch(k_rbgs_tma2<T, TPR, CP, TY, D, true>, ntiles, NT, SM, st, bl, tiles, zc, maps, rmaps, dst, fx, fy, fz, err, om);
  else pdl_launch(k_rbgs_tma2<T, TPR, CP, TY, D, false>, ntiles, NT, SM, st, bl, tiles, zc, maps, rmaps, dst, fx, fy, fz, err, om);
  return cudaGetLastError();
}

// (variant, threads per row, pairs per thread, rows, prefetch depth)
#define H3D_TMA2_SHAPES(X) \
  X(19, 32, 2, 4, 3)       \
  X(20, 32, 2, 8, 3)       \
  X(21, 64, 1, 4, 3)       \
  X(22, 64, 1, 8, 3)       \
  X(23, 32, 1, 8, 3)       \
  X(24, 32, 1, 16, 2)      \
  X(25, 16, 1, 16, 2)      \
  X(26, 32, 2, 16, 2)      \
  X(27, 32, 2, 8, 2)       \
  X(28, 8, 1, 16, 2)

// One cell of the seven-point update, over-relaxed: (rhs - off-diagonal sum) x
// (omega x diagonal reciprocal) + (1 - omega) x old value, one FMA (omega = 1:
// the Gauss-Seidel value exactly).
__device__ __forceinline__ float win_upd(float w, float e, float s, float n, float b, float t, float rv, float aw,
                                         float ae, float as, float an, float ab, float at, float iv, float old,
                                         float omc) {
  const float sum = fmaf(at, t, fmaf(ab, b, fmaf(an, n, fmaf(as, s, fmaf(ae, e, aw * w)))));
  return fmaf(rv - sum, iv, omc * old);
}

// The two cells of one colour of a group of four (positions 0, 2 when q1 is
// false, else 1, 3).  aw0 / iv0 belong to the first cell of the group, ae3 /
// iv3 to the last, iv12 to the middle two; the reciprocals carry omega,
// omc = 1 - omega.
__device__ __forceinline__ void win_colour(float4& c, const float4& bz, const float4& tz, const float4& u,
                                           const float4& dn, const float4& rh, float l, float r, bool q1, float aw0,
                                           float ae3, float ax, float as, float an, float ab, float at, float iv0,
                                           float iv12, float iv3, float omc) {
  if (!q1) {
    c.x = win_upd(l, c.y, u.x, dn.x, bz.x, tz.x, rh.x, aw0, ax, as, an, ab, at, iv0, c.x, omc);
    c.z = win_upd(c.y, c.w, u.z, dn.z, bz.z, tz.z, rh.z, ax, ax, as, an, ab, at, iv12, c.z, omc);
  } else {
    c.y = win_upd(c.x, c.z, u.y, dn.y, bz.y, tz.y, rh.y, ax, ax, as, an, ab, at, iv12, c.y, omc);
    c.w = win_upd(c.z, r, u.w, dn.w, bz.w, tz.w, rh.w, ax, ae3, as, an, ab, at, iv3, c.w, omc);
  }
}

// ---------------------------------------------------------------------------
// Register-window TMA sweep (k_rbgs_win), FP32 with constant coefficients.
//
// Same phases, staging and results as k_rbgs_vec, but a thread keeps its own
// GPT groups of four cells (x0 = 1 + 4g, g = j + k*TPR) of planes z-3 .. z+1
// in registers for the whole z march, so a phase reads from shared memory
// only the groups of the new plane z+1, the rows y-1 and y+1 at planes z
// (red) and z-2 (black) and the right-hand side; the cells left and right of
// a group come from the neighbouring lanes by warp shuffles (a row is TPR
// consecutive lanes), the ghost columns from shared memory.  A plane is last
// read two phases after its own, so the ring needs D+3 slots.  ZERO: the
// source iterate is identically zero (first sweep of a cycle): only the
// right-hand side is staged, red cells are rhs times the diagonal reciprocal,
// and black cells read the red values of neighbours in the block (zero
// outside it).  GPT = 2 halves the per-plane overhead per cell.
template <int TPR, int GPT, int TY, int NS, int D, bool ZERO, int U>
__global__ void __launch_bounds__(TPR*(TY + 2)) k_rbgs_win(const BlkLev* __restrict__ bls,
                                                          const Tile* __restrict__ tiles, int zc,
                                                          const CUtensorMap* __restrict__ maps,
                                                          const CUtensorMap* __restrict__ rmaps,
                                                          float* __restrict__ dst, int* err,
                                                          const long long* __restrict__ push, float om) {
  pdl_trigger();
  using C = VecCfg<TPR, GPT, TY, NS, D>;
  static_assert(TPR <= 32 && (TPR & (TPR - 1)) == 0, "a row is a power-of-two lane segment of one warp");
  static_assert(GPT == 1 || GPT == 2, "one or two groups per lane");
  constexpr int R = TY + 2;         // rows of a tile with its two halo rows
  constexpr int RE = (R + 1) / 2;   // rows of even index within the tile
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_base128(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NS * C::SLOT);

  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const CUtensorMap* map = maps + t.b;
  const CUtensorMap* rmap = rmaps + t.b;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sxy = B.sxy;
  const int y0 = t.y0, zs = t.z0;
  const int ze = min(zs + zc - 1, nz);
  const int zlo = max(zs - 1, 1), zhi = min(ze + 1, nz);
  const int BX = (nx + 2 + kXOff + 3) & ~3;  // smem row pitch == TMA box width
  const uint32_t tx_bytes = (uint32_t)(BX * ((ZERO ? 0 : TY + 4) + TY + 2) * 4);
  // Lane segments hold rows of equal parity back to back (even rows first),
  // so a warp that holds several rows updates cells of one colour in a phase.
  const int seg = threadIdx.x / TPR, j = threadIdx.x % TPR;
  const int tr = TPR == 32 ? seg : (seg < RE ? 2 * seg : 2 * (seg - RE) + 1);
  const int y = y0 - 1 + tr;
  const bool yrow = y >= 1 && y <= ny;
  int x0[GPT], pc[GPT], rcol[GPT];
  bool gin[GPT], lft[GPT], rgt[GPT];
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    x0[k] = 1 + 4 * (j + k * TPR);
    gin[k] = x0[k] <= nx;
    lft[k] = x0[k] == 1;
    rgt[k] = x0[k] + 3 == nx;  // groups next to the ghost columns
    pc[k] = (tr + 1) * BX + kXOff + x0[k];  // own group in an iterate slot
    rcol[k] = tr * BX + kXOff + x0[k];      // own group in a right-hand-side slot
  }
  float* __restrict__ Drow = dst + B.off + (long long)y * B.sx;
  const bool leader = threadIdx.x == 0;
  bool bad = false;
  // ghost pushes: face f (W, E, S, N, B, T) of this block is the source of a
  // whole ghost face; its new values are also stored at their own address +
  // pd[f] (kNoPush: none), so the fill after the sweep skips those faces
  long long pd[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) pd[f] = push ? __ldg(push + 6 * t.b + f) : kNoPush;
  // which pushes this thread does: x faces at the row ends (every row), y faces
  // on the block's first and last rows (loop invariant), z faces on the
  // first and last planes (decided per plane, uniform over the CTA)
  bool pxw[GPT], pxe[GPT];
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    pxw[k] = lft[k] && pd[0] != kNoPush;
    pxe[k] = rgt[k] && pd[1] != kNoPush;
  }
  const bool pys = y == 1 && pd[2] != kNoPush, pyn = y == ny && pd[3] != kNoPush;
  const bool pzb = pd[4] != kNoPush, pzt = pd[5] != kNoPush;

  // constant coefficients (mgsolver.for:186-205): walls zero the face term
  const int ph = B.phys;
  const float ax = (float)B.ax, ay = (float)B.ay, az = (float)B.az;
  const float as = (y == 1 && (ph & 4)) ? 0.f : ay;
  const float an = (y == ny && (ph & 8)) ? 0.f : ay;
  float aw0[GPT], ae3[GPT];
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    aw0[k] = (lft[k] && (ph & 1)) ? 0.f : ax;
    ae3[k] = (rgt[k] && (ph & 2)) ? 0.f : ax;
  }
  // diagonal reciprocals (times omega) of the three kinds of cells of a group
  // on interior planes, the bottom wall plane (b), the top wall plane (t) and a
  // plane that is both (bt, nz = 1): no division inside the z march
  const float omc = 1.f - om;
  auto rcp = [&](float aw, float ae, float ab, float at) { return om * (1.f / (-(aw + ae + as + an + ab + at))); };
  float i0[GPT], i0b[GPT], i0t[GPT], i0bt[GPT], i3[GPT], i3b[GPT], i3t[GPT], i3bt[GPT];
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    i0[k] = rcp(aw0[k], ax, az, az);
    i0b[k] = rcp(aw0[k], ax, 0.f, az);
    i0t[k] = rcp(aw0[k], ax, az, 0.f);
    i0bt[k] = rcp(aw0[k], ax, 0.f, 0.f);
    i3[k] = rcp(ax, ae3[k], az, az);
    i3b[k] = rcp(ax, ae3[k], 0.f, az);
    i3t[k] = rcp(ax, ae3[k], az, 0.f);
    i3bt[k] = rcp(ax, ae3[k], 0.f, 0.f);
  }
  const float i12 = rcp(ax, ax, az, az), i12b = rcp(ax, ax, 0.f, az), i12t = rcp(ax, ax, az, 0.f),
              i12bt = rcp(ax, ax, 0.f, 0.f);

  if (leader) {
    for (int q = 0; q < NS; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + q)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  pdl_wait();  // everything above reads only setup data

  auto pslot = [&](int s) -> float* { return reinterpret_cast<float*>(base + s * C::SLOT); };
  auto rslot = [&](int s) -> const float* { return reinterpret_cast<const float*>(base + s * C::SLOT + C::PSLOT); };
  int last_q = -1;  // last plane issued (leader)
  auto issue = [&](int z) {  // leader only
    last_q = z;
    const int sl = (int)((unsigned)z % (unsigned)NS);
    const uint32_t bar = smem_u32(bars + sl);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    if (!ZERO)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
              "r"(smem_u32(pslot(sl))),
          "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y0 - 2), "r"(z), "r"(bar)
          : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(rslot(sl))),
        "l"(reinterpret_cast<uint64_t>(rmap)), "r"(0), "r"(y0 - 1), "r"(z), "r"(bar)
        : "memory");
  };
  // plane z sits in slot sl; it is the ((z - zlo + 1) / NS)-th use of that slot
  auto wait_plane = [&](int sl, int z) {
    const uint32_t parity = ((unsigned)(z - zlo + 1) / (unsigned)NS) & 1u;
    mbar_wait(smem_u32(bars + sl), parity, err, bad);
  };
  // ring slot of i in [-NS, 2 NS): a mask when the ring is a power of two
  auto wrap = [](int i) {
    if constexpr ((NS & (NS - 1)) == 0) return i & (NS - 1);
    else return i < 0 ? i + NS : (i >= NS ? i - NS : i);
  };
  // Cells of colour q1 (positions q1, q1+2) of group k (c) in plane z, with
  // the group below (bz) and above (tz), rows y-1 (u) and y+1 (dn), rhs rh,
  // and the cells left (l) and right (r) of the group.  Planes off the walls
  // (all but at most two) take the branch with the interior coefficients; the
  // branch is uniform over the CTA.
#define H3D_WIN_COLOUR(c, bz, tz, u, dn, rh, l, r, zz, q1, k)                                                    \
  do {                                                                                                           \
    const bool wlo_ = (zz) == 1 && (ph & 16), whi_ = (zz) == nz && (ph & 32);                                    \
    if (!(wlo_ || whi_)) {                                                                                       \
      win_colour(c, bz, tz, u, dn, rh, l, r, q1, aw0[k], ae3[k], ax, as, an, az, az, i0[k], i12, i3[k], omc);     \
    } else {                                                                                                     \
      win_colour(c, bz, tz, u, dn, rh, l, r, q1, aw0[k], ae3[k], ax, as, an, wlo_ ? 0.f : az, whi_ ? 0.f : az,   \
                 wlo_ ? (whi_ ? i0bt[k] : i0b[k]) : (whi_ ? i0t[k] : i0[k]),                                     \
                 wlo_ ? (whi_ ? i12bt : i12b) : (whi_ ? i12t : i12),                                             \
                 wlo_ ? (whi_ ? i3bt[k] : i3b[k]) : (whi_ ? i3t[k] : i3[k]), omc);                               \
    }                                                                                                            \
  } while (0)
  auto ld4 = [](const float* p) { return *reinterpret_cast<const float4*>(p); };
  // lanes of this warp that exist (the last warp of a CTA can be partial)
  constexpr bool kWholeWarps = (TPR * R) % 32 == 0;
  const int wlanes = min(32, (int)blockDim.x - (int)(threadIdx.x & ~31u));
  const unsigned FULL = kWholeWarps ? 0xffffffffu : (wlanes == 32 ? 0xffffffffu : ((1u << wlanes) - 1u));
  // Cells left (.w of the group before) and right (.x of the group after) of
  // every group k, from the neighbouring lanes of the row (ghost columns and
  // a zero source outside the row are handled by the caller).
  auto sides = [&](const float4 (&g)[GPT], float (&l)[GPT], float (&r)[GPT]) {
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      l[k] = __shfl_up_sync(FULL, g[k].w, 1, TPR);
      r[k] = __shfl_down_sync(FULL, g[k].x, 1, TPR);
    }
    if (GPT == 2) {  // across the two halves of the row: group TPR-1 <-> group TPR
      const float lw = __shfl_sync(FULL, g[0].w, TPR - 1, TPR);
      const float rx = __shfl_sync(FULL, g[GPT - 1].x, 0, TPR);
      if (j == 0) l[GPT - 1] = lw;
      if (j == TPR - 1) r[0] = rx;
    }
  };

  if (leader)
    for (int q = zlo - 1; q <= min(zlo + D, zhi + 1); ++q) issue(q);
  int s0 = (int)((unsigned)zlo % (unsigned)NS);  // slot of plane z
  wait_plane(wrap(s0 - 1), zlo - 1);
  wait_plane(s0, zlo);
  // own groups of planes z-3 .. z+1 (planes below z hold their red updates)
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 m3[GPT], m2[GPT], m1[GPT], c0[GPT], p1[GPT];
#pragma unroll
  for (int k = 0; k < GPT; ++k) {
    m3[k] = zero4;
    m2[k] = zero4;
    p1[k] = zero4;
    m1[k] = ZERO ? zero4 : ld4(pslot(wrap(s0 - 1)) + pc[k]);
    c0[k] = ZERO ? zero4 : ld4(pslot(s0) + pc[k]);
  }
  long long dz = (long long)(zlo - 2) * sxy;  // offset of plane z-2 in the block
#pragma unroll U
  for (int z = zlo; z <= ze + 2; ++z, dz += sxy) {
    const int zb = z - 2;
    const bool red = z <= zhi && yrow;                                // red cells of plane z
    const bool blk = zb >= zs && zb <= ze && yrow && tr >= 1 && tr <= TY;  // black cells of plane z-2
    const bool q1 = (y + z) & 1;  // red cells of plane z at positions 1, 3 of the groups
    float* Pz = pslot(s0);
    const float* Rz = rslot(s0);
    const int sb = wrap(s0 - 2);
    const float* Pb = pslot(sb);
    const float* Rb = rslot(sb);
    if (z <= zhi) {
      const int sp = wrap(s0 + 1);
      wait_plane(sp, z + 1);
      if (!ZERO) {
#pragma unroll
        for (int k = 0; k < GPT; ++k) p1[k] = ld4(pslot(sp) + pc[k]);
      }
    }
    float rl[GPT], rr[GPT], bl[GPT], br[GPT];
    sides(c0, rl, rr);
    sides(m2, bl, br);
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      if (red && gin[k]) {
        const float4 h = ld4(Rz + rcol[k]);
        float4 u = zero4, dn = zero4;
        if (!ZERO) {
          u = ld4(Pz + pc[k] - BX);
          dn = ld4(Pz + pc[k] + BX);
          if (lft[k]) rl[k] = Pz[pc[k] - 1];
          if (rgt[k]) rr[k] = Pz[pc[k] + 4];
        }
        H3D_WIN_COLOUR(c0[k], m1[k], p1[k], u, dn, h, rl[k], rr[k], z, q1, k);
        *reinterpret_cast<float4*>(Pz + pc[k]) = c0[k];
      }
    }
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      if (blk && gin[k]) {
        const float4 h = ld4(Rb + rcol[k]);
        float4 u = zero4, dn = zero4;
        if (!ZERO) {
          u = ld4(Pb + pc[k] - BX);
          dn = ld4(Pb + pc[k] + BX);
          if (lft[k]) bl[k] = Pb[pc[k] - 1];
          if (rgt[k]) br[k] = Pb[pc[k] + 4];
        } else {  // red neighbours inside the block; the zero source outside it
          if (y > 1) u = ld4(Pb + pc[k] - BX);
          if (y < ny) dn = ld4(Pb + pc[k] + BX);
          if (lft[k]) bl[k] = 0.f;
          if (rgt[k]) br[k] = 0.f;
        }
        H3D_WIN_COLOUR(m2[k], m3[k], m1[k], u, dn, h, bl[k], br[k], zb, !q1, k);
        float* o = Drow + dz + x0[k];
        *reinterpret_cast<float4*>(o) = m2[k];
        if (pxw[k]) o[pd[0]] = m2[k].x;
        if (pxe[k]) o[3 + pd[1]] = m2[k].w;
        const bool pz = (zb == 1 && pzb) || (zb == nz && pzt);
        if (__builtin_expect(pys || pyn || pz, 0)) {  // rare: two rows and two planes of a block
          if (pys) *reinterpret_cast<float4*>(o + pd[2]) = m2[k];
          if (pyn) *reinterpret_cast<float4*>(o + pd[3]) = m2[k];
          if (zb == 1 && pzb) *reinterpret_cast<float4*>(o + pd[4]) = m2[k];
          if (zb == nz && pzt) *reinterpret_cast<float4*>(o + pd[5]) = m2[k];
        }
      }
    }
    // this phase's shared-memory writes are ordered before the TMA that reuses their slot
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (leader && !bad && z + D + 1 <= zhi + 1) issue(z + D + 1);
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      m3[k] = m2[k];
      m2[k] = m1[k];
      m1[k] = c0[k];
      c0[k] = p1[k];
    }
    s0 = wrap(s0 + 1);
  }
  if (leader && bad) drain_ring(bars, NS, zlo - 1, last_q, err);
}

#undef H3D_WIN_COLOUR

template <int TPR, int GPT, int TY, int NS, int D>
static cudaError_t vec_attr() {
  return cudaFuncSetAttribute(k_rbgs_vec<TPR, GPT, TY, NS, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VecCfg<TPR, GPT, TY, NS, D>::SMEM);
}

template <int TPR, int GPT, int TY, int NS, int D>
static cudaError_t vec_dispatch(const BlkLev* bl, const Tile* tiles, int ntiles, int zc, const CUtensorMap* maps,
                                const CUtensorMap* rmaps, int* err, float* dst, float om, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  pdl_launch(k_rbgs_vec<TPR, GPT, TY, NS, D>, ntiles, TPR * (TY + 2), VecCfg<TPR, GPT, TY, NS, D>::SMEM, st, 
      bl, tiles, zc, maps, rmaps, dst, err, om);
  return cudaGetLastError();
}

template <int TPR, int GPT, int TY, int NS, int D, int U>
static cudaError_t win_attr() {
  cudaError_t e = cudaFuncSetAttribute(k_rbgs_win<TPR, GPT, TY, NS, D, false, U>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)VecCfg<TPR, GPT, TY, NS, D>::SMEM);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_rbgs_win<TPR, GPT, TY, NS, D, true, U>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VecCfg<TPR, GPT, TY, NS, D>::SMEM);
}

template <int TPR, int GPT, int TY, int NS, int D, int U>
static cudaError_t win_dispatch(bool zero, const BlkLev* bl, const Tile* tiles, int ntiles, int zc,
                                const CUtensorMap* maps, const CUtensorMap* rmaps, int* err, float* dst,
                                const long long* push, float om, cudaStream_t st) {
  static_assert(D + 3 <= NS, "a plane is read until two phases after its own");
  if (ntiles <= 0) return cudaSuccess;
  constexpr size_t SM = VecCfg<TPR, GPT, TY, NS, D>::SMEM;
  if (zero)
    pdl_launch(k_rbgs_win<TPR, GPT, TY, NS, D, true, U>, ntiles, TPR * (TY + 2), SM, st, bl, tiles, zc, maps, rmaps,
               dst, err, push, om);
  else
    pdl_launch(k_rbgs_win<TPR, GPT, TY, NS, D, false, U>, ntiles, TPR * (TY + 2), SM, st, bl, tiles, zc, maps, rmaps,
               dst, err, push, om);
  return cudaGetLastError();
}

constexpr int kFirstWinShape = 40;
// (variant, lanes per row, groups of four cells per lane, rows, ring slots, prefetch depth,
//  z-march unrolling: 5 = the length of the register window, so that it rotates without moves)
#define H3D_WIN_SHAPES(X)     \
  X(40, 32, 1, 4, 8, 5, 1)    \
  X(41, 32, 1, 8, 8, 4, 1)    \
  X(42, 32, 1, 16, 8, 4, 1)   \
  X(43, 32, 1, 8, 8, 5, 1)    \
  X(44, 16, 1, 8, 8, 5, 1)    \
  X(45, 16, 1, 16, 8, 4, 1)   \
  X(46, 8, 1, 16, 8, 5, 1)    \
  X(47, 4, 1, 16, 8, 5, 1)    \
  X(48, 16, 2, 16, 8, 4, 1)   \
  X(49, 16, 2, 8, 8, 4, 1)    \
  X(50, 8, 2, 16, 8, 4, 1)    \
  X(51, 32, 1, 8, 8, 4, 5)    \
  X(52, 32, 1, 16, 8, 4, 5)   \
  X(53, 32, 1, 8, 8, 5, 5)    \
  X(54, 16, 1, 8, 8, 5, 5)    \
  X(55, 16, 1, 16, 8, 4, 5)   \
  X(56, 8, 1, 16, 8, 5, 5)    \
  X(57, 16, 2, 8, 8, 4, 5)    \
  X(58, 32, 1, 4, 8, 5, 5)    \
  X(59, 32, 1, 15, 8, 4, 5)   \
  X(60, 32, 1, 15, 8, 5, 5)

// (variant, threads per row, groups of four cells per thread, rows, ring slots, prefetch depth)
#define H3D_VEC_SHAPES(X)  \
  X(30, 32, 1, 4, 8, 4)    \
  X(31, 32, 1, 8, 8, 4)    \
  X(32, 32, 1, 8, 6, 2)    \
  X(33, 32, 1, 16, 6, 2)   \
  X(34, 16, 2, 8, 6, 2)    \
  X(35, 16, 2, 16, 6, 2)   \
  X(36, 16, 1, 8, 8, 4)    \
  X(37, 16, 1, 16, 6, 2)   \
  X(38, 8, 1, 16, 6, 2)    \
  X(39, 4, 1, 16, 6, 2)

#define H3D_ROW_SHAPES(X)  \
  X(8, 64, 1, 8)           \
  X(9, 32, 2, 8)           \
  X(10, 32, 1, 8)          \
  X(11, 32, 1, 16)         \
  X(12, 16, 1, 16)         \
  X(13, 8, 1, 16)          \
  X(14, 64, 2, 8)          \
  X(15, 64, 1, 4)          \
  X(16, 128, 1, 4)         \
  X(17, 32, 2, 4)          \
  X(18, 32, 4, 8)          \
  X(29, 32, 2, 16)

cudaError_t defect_march_attributes();
cudaError_t coarse_tail_attributes();

cudaError_t init_kernel_attributes() {
  cudaError_t e = cudaSuccess;
#define X(v, tpr, cp, ty)                                                  \
  if ((e = rows_attr<float, tpr, cp, ty>()) != cudaSuccess) return e;      \
  if ((e = rows_attr<double, tpr, cp, ty>()) != cudaSuccess) return e;
  H3D_ROW_SHAPES(X)
#undef X
#define X(v, tpr, cp, ty, d)                                                 \
  if ((e = tma2_attr<float, tpr, cp, ty, d>()) != cudaSuccess) return e;     \
  if ((e = tma2_attr<double, tpr, cp, ty, d>()) != cudaSuccess) return e;
  H3D_TMA2_SHAPES(X)
#undef X
#define X(v, tpr, gpt, ty, ns, d) \
  if ((e = vec_attr<tpr, gpt, ty, ns, d>()) != cudaSuccess) return e;
  H3D_VEC_SHAPES(X)
#undef X
#define X(v, tpr, gpt, ty, ns, d, u) \
  if ((e = win_attr<tpr, gpt, ty, ns, d, u>()) != cudaSuccess) return e;
  H3D_WIN_SHAPES(X)
#undef X
  cudaError_t e2 = defect_march_attributes();
  if (e2 != cudaSuccess) return e2;
  return coarse_tail_attributes();
}



bool rbgs_pushes(int variant, bool var, bool f32) {
  return f32 && !var && variant >= kFirstWinShape && variant < num_tile_shapes();
}

template <typename T>
cudaError_t launch_rbgs(int variant, bool var, bool zero_src, const BlkLev* bl, const Tile* tiles, int ntiles,
                        int zc, const CUtensorMap* maps, const CUtensorMap* rmaps, int* err, const T* src, T* dst,
                        const T* rhs, const T* fx, const T* fy, const T* fz, const long long* push, float om,
                        cudaStream_t st) {
  // ghost pushes need the register-window sweep to run as asked
  if (push && (!rbgs_pushes(variant, var, sizeof(T) == 4) || !maps || !rmaps)) return cudaErrorInvalidValue;
  if (variant >= 0 && variant < num_tile_shapes() && kShapes[variant].tma) {
    // nothing to stage from a zero source: the equivalent plain-load kernel zero-fills;
    // the vectorised sweep is FP32 with constant coefficients only
    const int tk = kShapes[variant].tma;
    const bool win = variant >= kFirstWinShape;  // register-window sweeps handle a zero source themselves
    if ((zero_src && !(win && sizeof(T) == 4 && !var)) || !maps || (tk >= 2 && !rmaps) ||
        (tk == 3 && (var || sizeof(T) != 4)))
      variant = kShapes[variant].alt;
  }
  if constexpr (sizeof(T) == 4) {
    switch (variant) {
#define X(v, tpr, gpt, ty, ns, d) \
      case v: return vec_dispatch<tpr, gpt, ty, ns, d>(bl, tiles, ntiles, zc, maps, rmaps, err, reinterpret_cast<float*>(dst), om, st);
      H3D_VEC_SHAPES(X)
#undef X
#define X(v, tpr, gpt, ty, ns, d, u) \
      case v: return win_dispatch<tpr, gpt, ty, ns, d, u>(zero_src, bl, tiles, ntiles, zc, maps, rmaps, err, reinterpret_cast<float*>(dst), push, om, st);
      H3D_WIN_SHAPES(X)
#undef X
      default: break;
    }
  }
  switch (variant) {
    case 0: return rbgs_dispatch<T, 32, 16, 256>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 1: return rbgs_dispatch<T, 32, 8, 256>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 2: return rbgs_dispatch<T, 64, 8, 256>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 3: return rbgs_dispatch<T, 16, 8, 128>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 4: return rbgs_dispatch<T, 8, 8, 64>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 5: return rbgs_dispatch<T, 8, 4, 32>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 6: return rbgs_dispatch<T, 4, 4, 32>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    case 7: return rbgs_dispatch<T, 64, 16, 512>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
#define X(v, tpr, cp, ty) \
    case v: return rows_dispatch<T, tpr, cp, ty>(var, zero_src, bl, tiles, ntiles, zc, src, dst, rhs, fx, fy, fz, om, st);
    H3D_ROW_SHAPES(X)
#undef X
#define X(v, tpr, cp, ty, d) \
    case v: return tma2_dispatch<T, tpr, cp, ty, d>(var, bl, tiles, ntiles, zc, maps, rmaps, err, dst, fx, fy, fz, om, st);
    H3D_TMA2_SHAPES(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// Several sweeps of a small level (mgrelax with `sweeps` iterations) in one
// CTA, in place: per sweep the red cells (x+y+z odd), a barrier, the black
// cells, a barrier, then the ghost fill from the level's sweep table (every
// entry reads an interior cell, so the gather is order-free in place), a
// barrier.  Same cell values as the out-of-place sweep + fill kernels: the
// FP64 update keeps the reference's operand order and IEEE division.
// zero: the iterate is known zero; it is cleared (ghosts included) first.
// start[b]: first flat interior index of block b (start[nb] = all cells).
// sb / ss: the block table and those starts, in shared memory.
template <typename T, bool VAR>
__device__ void small_relax(const BlkLev* sb, const int* ss, int nb, T* __restrict__ phi, const T* __restrict__ rhs,
                            const T* __restrict__ fx, const T* __restrict__ fy, const T* __restrict__ fz,
                            const uint32_t* __restrict__ fdst, const uint32_t* __restrict__ fsrc, int nfill,
                            int sweeps, int zero, long long nelems, float om, int rb) {
  const int ncell = ss[nb];
  if (zero) {
    for (long long q = threadIdx.x; q < nelems; q += blockDim.x) phi[q] = T(0);
    __syncthreads();
  }
  for (int it = 0; it < sweeps; ++it) {
    for (int colour = 1; colour >= 0; --colour) {  // red (x+y+z odd) first
      for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
        int b = 0;
        while (b + 1 < nb && ss[b + 1] <= c) ++b;
        const BlkLev& B = sb[b];
        const int local = c - ss[b];
        const int x = 1 + local % B.nx, y = 1 + (local / B.nx) % B.ny, z = 1 + local / (B.nx * B.ny);
        if (((x + y + z) & 1) != colour) continue;
        const long long i = B.off + (long long)z * B.sxy + (long long)y * B.sx + x;
        const Coef<T> cf = cell_coef<T, VAR>(B, x, y, z, i - B.off, VAR ? fx + B.off : nullptr,
                                             VAR ? fy + B.off : nullptr, VAR ? fz + B.off : nullptr);
        const T ap = coef_ap(cf);
        T v = gs_div(rhs[i] - (cf.aw * phi[i - 1] + cf.ae * phi[i + 1] + cf.as * phi[i - B.sx] +
                               cf.an * phi[i + B.sx] + cf.ab * phi[i - B.sxy] + cf.at * phi[i + B.sxy]),
                     ap);
        if constexpr (sizeof(T) == 4) v = sorf(phi[i], v, om);
        phi[i] = v;
      }
      __syncthreads();
      if (rb && colour == 1) {  // red-black order across block faces: the new red cells into the ghosts
        for (int q = threadIdx.x; q < nfill; q += blockDim.x) phi[fdst[q]] = phi[fsrc[q] & kIdxMask];
        __syncthreads();
      }
    }
    for (int q = threadIdx.x; q < nfill; q += blockDim.x) phi[fdst[q]] = phi[fsrc[q] & kIdxMask];
    __syncthreads();
  }
}

// All sweeps of one relaxation visit of a level whose ghost fill stays inside
// every block (independent blocks, a single block, periodic wraps onto
// itself): one CTA per block, in place, the cell arithmetic of small_relax;
// fill entries of block b are fstart[b] .. fstart[b+1]-1 (sources in block b).
template <typename T, bool VAR>
__global__ void __launch_bounds__(1024) k_relax_blocks(const BlkLev* __restrict__ bls, const int* __restrict__ fstart,
                                                       T* __restrict__ phi, const T* __restrict__ rhs,
                                                       const T* __restrict__ fx, const T* __restrict__ fy,
                                                       const T* __restrict__ fz, const uint32_t* __restrict__ fdst,
                                                       const uint32_t* __restrict__ fsrc, int sweeps, int zero,
                                                       float om) {
  pdl_trigger();
  const BlkLev B = bls[blockIdx.x];
  const int f0 = fstart[blockIdx.x], f1 = fstart[blockIdx.x + 1];
  pdl_wait();
  if (zero) {
    const long long n = (long long)(B.nz + 2) * B.sxy;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) phi[B.off + q] = T(0);
    __syncthreads();
  }
  const int ncell = B.nx * B.ny * B.nz;
  for (int it = 0; it < sweeps; ++it) {
    for (int colour = 1; colour >= 0; --colour) {  // red (x+y+z odd) first
      for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
        const int x = 1 + c % B.nx, y = 1 + (c / B.nx) % B.ny, z = 1 + c / (B.nx * B.ny);
        if (((x + y + z) & 1) != colour) continue;
        const long long i = B.off + (long long)z * B.sxy + (long long)y * B.sx + x;
        const Coef<T> cf = cell_coef<T, VAR>(B, x, y, z, i - B.off, VAR ? fx + B.off : nullptr,
                                             VAR ? fy + B.off : nullptr, VAR ? fz + B.off : nullptr);
        const T ap = coef_ap(cf);
        T v = gs_div(rhs[i] - (cf.aw * phi[i - 1] + cf.ae * phi[i + 1] + cf.as * phi[i - B.sx] +
                               cf.an * phi[i + B.sx] + cf.ab * phi[i - B.sxy] + cf.at * phi[i + B.sxy]),
                     ap);
        if constexpr (sizeof(T) == 4) v = sorf(phi[i], v, om);
        phi[i] = v;
      }
      __syncthreads();
    }
    for (int q = f0 + threadIdx.x; q < f1; q += blockDim.x) phi[fdst[q]] = phi[fsrc[q] & kIdxMask];
    __syncthreads();
  }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(1024) k_relax_small(const BlkLev* __restrict__ bls, const int* __restrict__ start,
                                                      int nb, T* __restrict__ phi, const T* __restrict__ rhs,
                                                      const T* __restrict__ fx, const T* __restrict__ fy,
                                                      const T* __restrict__ fz, const uint32_t* __restrict__ fdst,
                                                      const uint32_t* __restrict__ fsrc, int nfill, int sweeps,
                                                      int zero, long long nelems, float om, int rb) {
  pdl_trigger();
  __shared__ BlkLev sb[kSmallLevelBlocks];
  __shared__ int ss[kSmallLevelBlocks + 1];
  // the block table and cell starts are written once at setup: read them
  // while the predecessor finishes
  for (int b = threadIdx.x; b < nb; b += blockDim.x) sb[b] = bls[b];
  for (int b = threadIdx.x; b <= nb; b += blockDim.x) ss[b] = start[b];
  pdl_wait();
  __syncthreads();
  small_relax<T, VAR>(sb, ss, nb, phi, rhs, fx, fy, fz, fdst, fsrc, nfill, sweeps, zero, nelems, om, rb);
}

// The fused coarse tail keeps every tail level in shared memory, in a
// compact layout: the iterate as the padded blocks back to back (block b at
// cbl[b].off, pitches nx+2 and (nx+2)(ny+2)), the rhs as the interior cells
// in natural order (block b from cbl[b].pad).  Cells come from per-level
// tables built at setup, one 64-bit entry a cell: compact index (bits 0-23),
// x, y, z (bits 24-31, 32-39, 40-47) and block (bits 48-53); interior
// tables list the red cells (x+y+z odd) first.
struct CellRef {
  int i, x, y, z, b;
};
__device__ __forceinline__ CellRef cell_ref(unsigned long long e) {
  CellRef c;
  c.i = (int)(e & 0xffffffull);
  c.x = (int)((e >> 24) & 0xff);
  c.y = (int)((e >> 32) & 0xff);
  c.z = (int)((e >> 40) & 0xff);
  c.b = (int)((e >> 48) & 0x3f);
  return c;
}
__device__ __forceinline__ int rhs_index(const BlkLev& B, int x, int y, int z) {
  return B.pad + ((z - 1) * B.ny + (y - 1)) * B.nx + (x - 1);
}
__device__ __forceinline__ long long global_index(const BlkLev& G, int x, int y, int z) {
  return G.off + (long long)z * G.sxy + (long long)y * G.sx + x;
}

// The red then the black cells of one in-place sweep of a tail level; same
// cell arithmetic as small_relax.
template <typename T>
__device__ void tail_colours(const BlkLev* cb, const TailLevel& L, T* phi, const T* rhs, int only = -1) {
  for (int colour = 0; colour < 2; ++colour) {  // red (x+y+z odd) first
    if (only >= 0 && colour != only) continue;
    const int k0 = colour ? L.nred : 0, k1 = colour ? L.nint : L.nred;
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const CellRef c = cell_ref(L.cells[k]);
      const BlkLev& B = cb[c.b];
      const int i = c.i;
      const Coef<T> cf = cell_coef<T, false>(B, c.x, c.y, c.z, i - B.off, nullptr, nullptr, nullptr);
      const T ap = coef_ap(cf);
      T v = gs_div(rhs[rhs_index(B, c.x, c.y, c.z)] -
                       (cf.aw * phi[i - 1] + cf.ae * phi[i + 1] + cf.as * phi[i - B.sx] +
                        cf.an * phi[i + B.sx] + cf.ab * phi[i - B.sxy] + cf.at * phi[i + B.sxy]),
                   ap);
      if constexpr (sizeof(T) == 4) v = sorf(phi[i], v, L.om);
      phi[i] = v;
    }
    __syncthreads();
  }
}

// `sweeps` in-place red-black sweeps of a tail level, each followed by its
// ghost fill.
template <typename T>
__device__ void tail_relax(const BlkLev* cb, const TailLevel& L, T* phi, const T* rhs, int sweeps) {
  for (int it = 0; it < sweeps; ++it) {
    if (L.rb_global) {  // a fill after each colour: the red-black order across block faces
      for (int colour = 0; colour < 2; ++colour) {
        tail_colours<T>(cb, L, phi, rhs, colour);
        for (int q = threadIdx.x; q < L.nfill; q += blockDim.x) phi[L.fdst[q]] = phi[L.fsrc[q]];
        __syncthreads();
      }
      continue;
    }
    tail_colours<T>(cb, L, phi, rhs);
    for (int q = threadIdx.x; q < L.nfill; q += blockDim.x) phi[L.fdst[q]] = phi[L.fsrc[q]];
    __syncthreads();
  }
}

// mgrestr into a tail level: the same residual sum over the eight children,
// in the same order, as k_restrict; one thread a coarse cell.
template <typename T>
__device__ void tail_restrict(const BlkLev* fb, const BlkLev* cb, const TailLevel& Cl, const T* phi, const T* rhs,
                              T* rhs_c, int zero_fine) {
  for (int k = threadIdx.x; k < Cl.nint; k += blockDim.x) {
    const CellRef cc = cell_ref(Cl.cells[k]);
    const BlkLev& F = fb[cc.b];
    const int X = cc.x, Y = cc.y, Z = cc.z;
    const T* P = phi + F.off;
    T sum = T(0);
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const int x = 2 * X - 1 + di, y = 2 * Y - 1 + dj, z = 2 * Z - 1 + dk;
          const int i = z * (int)F.sxy + y * F.sx + x;
          const T rv = rhs[rhs_index(F, x, y, z)];
          T r;
          if (zero_fine) {
            r = rv - T(0);
          } else {
            Coef<T> cf = cell_coef<T, false>(F, x, y, z, i, nullptr, nullptr, nullptr);
            const T ap = coef_ap(cf);
            r = rv - (cf.aw * P[i - 1] + cf.ae * P[i + 1] + cf.as * P[i - F.sx] + cf.an * P[i + F.sx] +
                      cf.ab * P[i - F.sxy] + cf.at * P[i + F.sxy] + ap * P[i]);
          }
          sum = (di | dj | dk) ? sum + r : r;
        }
    rhs_c[rhs_index(cb[cc.b], X, Y, Z)] = T(0.125) * sum;
  }
  __syncthreads();
}

// mgcorr + mgbound of cell (x, y, z) (ghosts included) of block F: the value
// k_prolong writes there, reading the old iterate from `old`.
template <typename T>
__device__ __forceinline__ T tail_prolong_value(const BlkLev& F, const BlkLev& C, const T* phi_c, const T* old, int x,
                                                int y, int z, int zero_old) {
  const int ph = F.phys;
  int sx = x, sy = y, sz = z;
  if (x == 0 && (ph & 1)) sx = 1;
  if (x == F.nx + 1 && (ph & 2)) sx = F.nx;
  if (y == 0 && (ph & 4)) sy = 1;
  if (y == F.ny + 1 && (ph & 8)) sy = F.ny;
  if (z == 0 && (ph & 16)) sz = 1;
  if (z == F.nz + 1 && (ph & 32)) sz = F.nz;
  const T wx0 = (sx & 1) ? T(1) : T(3), wx1 = (sx & 1) ? T(3) : T(1);
  const T wy0 = (sy & 1) ? T(1) : T(3), wy1 = (sy & 1) ? T(3) : T(1);
  const T wz0 = (sz & 1) ? T(1) : T(3), wz1 = (sz & 1) ? T(3) : T(1);
  const int cy = C.sx, cz = (int)C.sxy;
  const T* Q = phi_c + C.off + (sz >> 1) * cz + (sy >> 1) * cy + (sx >> 1);
  // term order (di,dj,dk): 000, 010, 001, 011, 100, 110, 101, 111
  T s = (wx0 * wy0 * wz0) * Q[0];
  s = s + (wx0 * wy1 * wz0) * Q[cy];
  s = s + (wx0 * wy0 * wz1) * Q[cz];
  s = s + (wx0 * wy1 * wz1) * Q[cy + cz];
  s = s + (wx1 * wy0 * wz0) * Q[1];
  s = s + (wx1 * wy1 * wz0) * Q[1 + cy];
  s = s + (wx1 * wy0 * wz1) * Q[1 + cz];
  s = s + (wx1 * wy1 * wz1) * Q[1 + cy + cz];
  const T o = zero_old ? T(0) : old[F.off + sz * (int)F.sxy + sy * F.sx + sx];
  return o + s / T(64);
}

// mgcorr + mgbound into a tail level in place: the ghost cells read interior
// and ghost cells of the old iterate, so their new values go to `scratch`
// (one value a ghost-table entry) first; then the interior cells (each reads
// only itself) update in place, then the ghosts are copied back.
template <typename T>
__device__ void tail_prolong(const BlkLev* fb, const BlkLev* cb, const TailLevel& F, const T* phi_c, T* phi,
                             T* scratch, int zero_old) {
  for (int k = threadIdx.x; k < F.nghost; k += blockDim.x) {
    const CellRef c = cell_ref(F.ghosts[k]);
    scratch[k] = tail_prolong_value(fb[c.b], cb[c.b], phi_c, phi, c.x, c.y, c.z, zero_old);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < F.nint; k += blockDim.x) {
    const CellRef c = cell_ref(F.cells[k]);
    phi[c.i] = tail_prolong_value(fb[c.b], cb[c.b], phi_c, phi, c.x, c.y, c.z, zero_old);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < F.nghost; k += blockDim.x) phi[(int)(F.ghosts[k] & 0xffffffull)] = scratch[k];
  __syncthreads();
}

// The rhs of a tail level from global memory (the restriction into the
// first tail level ran outside); eight loads in flight a thread.
template <typename T>
__device__ void tail_load_rhs(const BlkLev* gb, const BlkLev* cb, const TailLevel& L, const T* __restrict__ g, T* rhs) {
  constexpr int U = 8;
  for (int k0 = threadIdx.x; k0 < L.nint; k0 += U * blockDim.x) {
    T v[U];
    int ri[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u * blockDim.x;
      ri[u] = -1;
      if (k < L.nint) {
        const CellRef c = cell_ref(L.cells[k]);
        v[u] = g[global_index(gb[c.b], c.x, c.y, c.z)];
        ri[u] = rhs_index(cb[c.b], c.x, c.y, c.z);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (ri[u] >= 0) rhs[ri[u]] = v[u];
  }
  __syncthreads();
}

// A tail level back to global memory: iterate (interior and ghost cells) and rhs.
template <typename T>
__device__ void tail_store(const BlkLev* gb, const BlkLev* cb, const TailLevel& L, const T* phi, const T* rhs,
                           T* __restrict__ gphi, T* __restrict__ grhs) {
  for (int k = threadIdx.x; k < L.nint + L.nghost; k += blockDim.x) {
    const CellRef c = cell_ref(k < L.nint ? L.cells[k] : L.ghosts[k - L.nint]);
    const long long gi = global_index(gb[c.b], c.x, c.y, c.z);
    gphi[gi] = phi[c.i];
    if (k < L.nint) grhs[gi] = rhs[rhs_index(cb[c.b], c.x, c.y, c.z)];
  }
  __syncthreads();
}

// The coarse end of a V-cycle in one CTA, every level in shared memory: the
// relaxations, restrictions, precision conversions and corrections of the
// tail levels run as the ops of a program built on the host, in order, with
// the CTA's barriers between them instead of kernel boundaries; one op loads
// the first tail level's rhs, the last ones store every tail level.
// curmask bit 2l (2l+1) selects the global FP32 (FP64) iterate buffer of
// tail level l.
__global__ void __launch_bounds__(1024) k_coarse_tail(const TailLevel* __restrict__ lv, const TailOp* __restrict__ ops,
                                                      int nops, unsigned curmask) {
  pdl_trigger();
  __shared__ BlkLev fb[kSmallLevelBlocks], cb[kSmallLevelBlocks], gb[kSmallLevelBlocks];
  extern __shared__ unsigned char smem_raw[];
  unsigned char* arena = smem_base128(smem_raw);
  pdl_wait();
  for (int o = 0; o < nops; ++o) {
    const TailOp op = ops[o];
    const TailLevel& F = lv[op.fine];
    const TailLevel& C = lv[op.coarse];
    const int nb = F.nb;
    __syncthreads();  // the previous op is done with the tables
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      fb[b] = F.cbl[b];
      cb[b] = C.cbl[b];
      gb[b] = F.gbl[b];
    }
    __syncthreads();
    auto at32 = [&](int off) { return reinterpret_cast<float*>(arena + off); };
    auto at64 = [&](int off) { return reinterpret_cast<double*>(arena + off); };
    switch (op.kind) {
      case kTailLoadRhs:
        if (op.f64) tail_load_rhs<double>(gb, fb, F, F.rhs64, at64(F.s_rhs64));
        else tail_load_rhs<float>(gb, fb, F, F.rhs32, at32(F.s_rhs32));
        break;
      case kTailRelax:
        if (op.f64) {
          double* phi = at64(F.s_phi64);
          if (op.zero) {
            for (int q = threadIdx.x; q < F.npad; q += blockDim.x) phi[q] = 0.0;
            __syncthreads();
          }
          tail_relax<double>(fb, F, phi, at64(F.s_rhs64), op.sweeps);
        } else {
          float* phi = at32(F.s_phi32);
          if (op.zero) {
            for (int q = threadIdx.x; q < F.npad; q += blockDim.x) phi[q] = 0.f;
            __syncthreads();
          }
          tail_relax<float>(fb, F, phi, at32(F.s_rhs32), op.sweeps);
        }
        break;
      case kTailRestrict:  // into the coarse rhs of the fine level's precision
        if (op.f64) tail_restrict<double>(fb, cb, C, at64(F.s_phi64), at64(F.s_rhs64), at64(C.s_rhs64), op.zero);
        else tail_restrict<float>(fb, cb, C, at32(F.s_phi32), at32(F.s_rhs32), at32(C.s_rhs32), op.zero);
        break;
      case kTailProlong:
        if (op.f64)
          tail_prolong<double>(fb, cb, F, at64(C.s_phi64), at64(F.s_phi64), at64(op.sweeps), op.zero);
        else
          tail_prolong<float>(fb, cb, F, at32(C.s_phi32), at32(F.s_phi32), at32(op.sweeps), op.zero);
        break;
      case kTailRhsF2D: {  // the coarsest rhs of a mixed solve to FP64
        const float* a = at32(F.s_rhs32);
        double* b = at64(F.s_rhs64);
        for (int q = threadIdx.x; q < F.nint; q += blockDim.x) b[q] = (double)a[q];
        __syncthreads();
        break;
      }
      case kTailPhiD2F: {  // the coarsest iterate of a mixed solve to FP32
        const double* a = at64(F.s_phi64);
        float* b = at32(F.s_phi32);
        for (int q = threadIdx.x; q < F.npad; q += blockDim.x) b[q] = (float)a[q];
        __syncthreads();
        break;
      }
      case kTailStore: {
        const int c32 = (curmask >> (2 * op.fine)) & 1, c64 = (curmask >> (2 * op.fine + 1)) & 1;
        if (F.s_phi32 >= 0) tail_store<float>(gb, fb, F, at32(F.s_phi32), at32(F.s_rhs32), F.phi32[c32], F.rhs32);
        if (F.s_phi64 >= 0) tail_store<double>(gb, fb, F, at64(F.s_phi64), at64(F.s_rhs64), F.phi64[c64], F.rhs64);
        break;
      }
      default:
        break;
    }
  }
}

// The coarse end of a V-cycle as one thread-block cluster: CTA b holds block
// b of every tail level in its shared memory (compact layout, every block of
// a level the same size) and runs the same op program as k_coarse_tail on
// it.  Restrictions, corrections and conversions only touch the CTA's own
// block; after the colours of a sweep the cluster synchronises, every CTA
// gathers its ghost cells from the other CTAs' shared memory (fdst: own
// compact index; fsrc: source rank << 24 | its compact index), and the
// cluster synchronises again before any interior changes.
__global__ void __launch_bounds__(kClusterTailThreads) k_coarse_cluster(const TailLevel* __restrict__ lvg,
                                                                        const TailOp* __restrict__ opsg, int nops,
                                                                        int nlev, unsigned curmask) {
  pdl_trigger();
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int b = (int)cl.block_rank();
  __shared__ TailLevel lv[kTailMaxLevels];
  __shared__ BlkLev gtab[kTailMaxLevels], ctab[kTailMaxLevels];  // this block per level: global / compact layout
  __shared__ TailOp ops[kClusterTailMaxOps];
  extern __shared__ unsigned char smem_raw[];
  unsigned char* arena = smem_base128(smem_raw);
  // the program, the level records and this block's tables are setup data:
  // stage them in shared memory (cell and ghost tables, this block's fill
  // entries) while the predecessor finishes
  for (int q = threadIdx.x; q < nops; q += blockDim.x) ops[q] = opsg[q];
  if (threadIdx.x < nlev) lv[threadIdx.x] = lvg[threadIdx.x];
  __syncthreads();
  for (int l = 0; l < nlev; ++l) {
    const TailLevel& G = lvg[l];
    unsigned long long* cs = reinterpret_cast<unsigned long long*>(arena + lv[l].s_cells);
    for (int k = threadIdx.x; k < G.nint + G.nghost; k += blockDim.x)
      cs[k] = k < G.nint ? __ldg(G.cells + k) : __ldg(G.ghosts + (k - G.nint));
    const int f0 = __ldg(G.fstart + b), f1 = __ldg(G.fstart + b + 1);
    uint32_t* fd = reinterpret_cast<uint32_t*>(arena + lv[l].s_fill);
    for (int k = threadIdx.x; k < f1 - f0; k += blockDim.x) {
      fd[2 * k] = __ldg(G.fdst + f0 + k);
      fd[2 * k + 1] = __ldg(G.fsrc + f0 + k);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      lv[l].cells = cs;
      lv[l].ghosts = cs + G.nint;
      lv[l].fdst = fd;
      lv[l].nfill = f1 - f0;
    }
  }
  __syncthreads();
  pdl_wait();
  auto compact = [](BlkLev B) {
    B.off = 0;
    B.sx = B.nx + 2;
    B.sxy = (long long)(B.nx + 2) * (B.ny + 2);
    B.pad = 0;
    return B;
  };
  if (threadIdx.x < nlev) {
    const BlkLev G = lvg[threadIdx.x].gbl[b];
    gtab[threadIdx.x] = G;
    ctab[threadIdx.x] = compact(G);
  }
  __syncthreads();
  for (int o = 0; o < nops; ++o) {
    const TailOp op = ops[o];
    const TailLevel& F = lv[op.fine];
    const TailLevel& C = lv[op.coarse];
    // this block's tables at the op's levels (staged once; every op ends with
    // a barrier of the CTA or the cluster)
    const BlkLev* gb = gtab + op.fine;
    const BlkLev* fb = ctab + op.fine;
    const BlkLev* cb = ctab + op.coarse;
    auto at32 = [&](int off) { return reinterpret_cast<float*>(arena + off); };
    auto at64 = [&](int off) { return reinterpret_cast<double*>(arena + off); };
    switch (op.kind) {
      case kTailLoadRhs:
        if (op.f64) tail_load_rhs<double>(gb, fb, F, F.rhs64, at64(F.s_rhs64));
        else tail_load_rhs<float>(gb, fb, F, F.rhs32, at32(F.s_rhs32));
        break;
      case kTailRelax: {
        auto relax = [&](auto* phi, const auto* rhs) {
          using T = typename std::remove_pointer<decltype(phi)>::type;
          if (op.zero) {
            for (int q = threadIdx.x; q < F.npad; q += blockDim.x) phi[q] = T(0);
            __syncthreads();
          }
          const int ncol = F.rb_global ? 2 : 1;  // 2: a fill after each colour (order across blocks)
          for (int it = 0; it < op.sweeps; ++it) {
            for (int pass = 0; pass < ncol; ++pass) {
              tail_colours<T>(fb, F, phi, rhs, ncol == 2 ? pass : -1);
              cl.sync();  // every block's sweep done
              for (int q = threadIdx.x; q < F.nfill; q += blockDim.x) {  // (dst, src) pairs of this block
                const uint32_t dsti = F.fdst[2 * q], src = F.fdst[2 * q + 1];
                const T* remote = cl.map_shared_rank(phi, (int)(src >> 24));
                phi[dsti] = remote[src & 0xffffffu];
              }
              cl.sync();  // every ghost gathered before any interior changes
            }
          }
        };
        if (op.f64) relax(at64(F.s_phi64), (const double*)at64(F.s_rhs64));
        else relax(at32(F.s_phi32), (const float*)at32(F.s_rhs32));
        break;
      }
      case kTailDense: {  // x = P b over the cells of every block (FP64), then the sweep fill
        double* phi = at64(F.s_phi64);
        const double* rhs = at64(F.s_rhs64);
        if (op.zero) {
          for (int q = threadIdx.x; q < F.npad; q += blockDim.x) phi[q] = 0.0;
        }
        cl.sync();  // every block's rhs is complete
        const int nper = F.nint, n = F.dense_n;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
        const BlkLev& B = fb[0];
        for (int i = warp; i < nper; i += nwarp) {  // a warp per row of this block; lanes split the columns
          const double* Pr = F.dense + (long long)(b * nper + i) * n;
          double s = 0.0;
          for (int j = lane; j < n; j += 32) {
            const double* r = cl.map_shared_rank(rhs, j / nper);
            s += __ldg(Pr + j) * r[j % nper];
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == 0) {
            const int x = i % B.nx + 1, y = (i / B.nx) % B.ny + 1, z = i / (B.nx * B.ny) + 1;
            phi[(long long)z * B.sxy + (long long)y * B.sx + x] = s;
          }
        }
        cl.sync();  // every block's interior is written
        for (int q = threadIdx.x; q < F.nfill; q += blockDim.x) {
          const uint32_t dsti = F.fdst[2 * q], src = F.fdst[2 * q + 1];
          const double* remote = cl.map_shared_rank(phi, (int)(src >> 24));
          phi[dsti] = remote[src & 0xffffffu];
        }
        cl.sync();  // every ghost gathered before any interior changes
        break;
      }
      case kTailRestrict:
        if (op.f64) tail_restrict<double>(fb, cb, C, at64(F.s_phi64), at64(F.s_rhs64), at64(C.s_rhs64), op.zero);
        else tail_restrict<float>(fb, cb, C, at32(F.s_phi32), at32(F.s_rhs32), at32(C.s_rhs32), op.zero);
        break;
      case kTailProlong:
        if (op.f64) tail_prolong<double>(fb, cb, F, at64(C.s_phi64), at64(F.s_phi64), at64(op.sweeps), op.zero);
        else tail_prolong<float>(fb, cb, F, at32(C.s_phi32), at32(F.s_phi32), at32(op.sweeps), op.zero);
        break;
      case kTailRhsF2D: {
        const float* x = at32(F.s_rhs32);
        double* y = at64(F.s_rhs64);
        for (int q = threadIdx.x; q < F.nint; q += blockDim.x) y[q] = (double)x[q];
        __syncthreads();
        break;
      }
      case kTailPhiD2F: {
        const double* x = at64(F.s_phi64);
        float* y = at32(F.s_phi32);
        for (int q = threadIdx.x; q < F.npad; q += blockDim.x) y[q] = (float)x[q];
        __syncthreads();
        break;
      }
      case kTailStore: {
        const int c32 = (curmask >> (2 * op.fine)) & 1, c64 = (curmask >> (2 * op.fine + 1)) & 1;
        if (F.s_phi32 >= 0) tail_store<float>(gb, fb, F, at32(F.s_phi32), at32(F.s_rhs32), F.phi32[c32], F.rhs32);
        if (F.s_phi64 >= 0) tail_store<double>(gb, fb, F, at64(F.s_phi64), at64(F.s_rhs64), F.phi64[c64], F.rhs64);
        break;
      }
      default:
        break;
    }
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

cudaError_t coarse_tail_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_coarse_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, kTailSmemBytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_coarse_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, kTailSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_coarse_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

static cudaError_t cluster_config(int nb, int smem_bytes, cudaStream_t st, cudaLaunchConfig_t* cfg,
                                  cudaLaunchAttribute* at) {
  *cfg = cudaLaunchConfig_t{};
  cfg->gridDim = dim3(nb);
  cfg->blockDim = dim3(kClusterTailThreads);
  cfg->dynamicSmemBytes = (size_t)smem_bytes;
  cfg->stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = nb;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg->attrs = at;
  cfg->numAttrs = 1;
  return cudaSuccess;
}

int coarse_cluster_fits(int nb, int smem_bytes) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[1];
  cluster_config(nb, smem_bytes, nullptr, &cfg, at);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_coarse_cluster, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

cudaError_t launch_coarse_cluster(int nb, const TailLevel* lv, int nlev, const TailOp* ops, int nops,
                                  unsigned curmask, int smem_bytes, cudaStream_t st) {
  if (nops <= 0 || nops > kClusterTailMaxOps || nlev > kTailMaxLevels) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[1];
  cluster_config(nb, smem_bytes, st, &cfg, at);
  return cudaLaunchKernelEx(&cfg, k_coarse_cluster, lv, ops, nops, nlev, curmask);
}

cudaError_t launch_coarse_tail(const TailLevel* lv, const TailOp* ops, int nops, unsigned curmask, int smem_bytes,
                               cudaStream_t st) {
  if (nops <= 0) return cudaSuccess;
  pdl_launch(k_coarse_tail, 1, 1024, (size_t)smem_bytes, st, lv, ops, nops, curmask);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_relax_small(bool var, const BlkLev* bl, const int* start, int nb, T* phi, const T* rhs,
                               const T* fx, const T* fy, const T* fz, const uint32_t* fdst, const uint32_t* fsrc,
                               int nfill, int sweeps, bool zero, long long nelems, float om, bool rb,
                               cudaStream_t st) {
  if (var)
    pdl_launch(k_relax_small<T, true>, 1, 1024, 0, st, bl, start, nb, phi, rhs, fx, fy, fz, fdst, fsrc, nfill, sweeps,
               (int)zero, nelems, om, (int)rb);
  else
    pdl_launch(k_relax_small<T, false>, 1, 1024, 0, st, bl, start, nb, phi, rhs, fx, fy, fz, fdst, fsrc, nfill,
               sweeps, (int)zero, nelems, om, (int)rb);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_relax_blocks(bool var, const BlkLev* bl, int nb, const int* fstart, T* phi, const T* rhs,
                                const T* fx, const T* fy, const T* fz, const uint32_t* fdst, const uint32_t* fsrc,
                                int sweeps, bool zero, float om, cudaStream_t st) {
  if (nb <= 0) return cudaSuccess;
  if (var)
    pdl_launch(k_relax_blocks<T, true>, nb, 1024, 0, st, bl, fstart, phi, rhs, fx, fy, fz, fdst, fsrc, sweeps,
               (int)zero, om);
  else
    pdl_launch(k_relax_blocks<T, false>, nb, 1024, 0, st, bl, fstart, phi, rhs, fx, fy, fz, fdst, fsrc, sweeps,
               (int)zero, om);
  return cudaGetLastError();
}
template cudaError_t launch_relax_blocks<double>(bool, const BlkLev*, int, const int*, double*, const double*,
                                                 const double*, const double*, const double*, const uint32_t*,
                                                 const uint32_t*, int, bool, float, cudaStream_t);
template cudaError_t launch_relax_blocks<float>(bool, const BlkLev*, int, const int*, float*, const float*,
                                                const float*, const float*, const float*, const uint32_t*,
                                                const uint32_t*, int, bool, float, cudaStream_t);
template cudaError_t launch_relax_small<double>(bool, const BlkLev*, const int*, int, double*, const double*,
                                                const double*, const double*, const double*, const uint32_t*,
                                                const uint32_t*, int, int, bool, long long, float, bool, cudaStream_t);
template cudaError_t launch_relax_small<float>(bool, const BlkLev*, const int*, int, float*, const float*,
                                               const float*, const float*, const float*, const uint32_t*,
                                               const uint32_t*, int, int, bool, long long, float, bool, cudaStream_t);

template <typename T>
cudaError_t launch_fill(const uint32_t* dsts, const uint32_t* srcs, int64_t n, T* out, const T* cur, const T* old,
                        bool zero_old, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int g = grid_for(n, 256);
  if (zero_old) pdl_launch(k_fill<T, true>, g, 256, 0, st, dsts, srcs, n, out, cur, old);
  else pdl_launch(k_fill<T, false>, g, 256, 0, st, dsts, srcs, n, out, cur, old);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Red values ahead of an FP32 sweep, for a red-black order across block faces.
// Inside one sweep a block's black cells read the cells across a block face
// from its ghost layer, which otherwise holds the values of before the sweep
// (the reference's order, mgsolver.for:614-615).  Entry e names a red
// interior cell src[e] of block blk[e] next to a face that another block (or a
// periodic partner) reads, and the ghost cell dst[e] that shows it there; the
// red update of src[e] is computed from the iterate (its six neighbours are
// black, still of before the sweep) and stored at dst[e], in place.  The
// block tables are staged in shared memory; info[e] carries the cell's block
// and wall faces, so no index arithmetic is needed.  With even
// block sizes a ghost cell of red colour is read by black cells only, so the
// sweep's red cells still see their old black neighbours, and no entry reads a
// cell another entry writes.
template <bool VAR>
__global__ void __launch_bounds__(256) k_red_ahead(const uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                                   const int* __restrict__ info, int64_t n, int nb,
                                                   const BlkLev* __restrict__ bls, float* __restrict__ phi,
                                                   const float* __restrict__ rhs, const float* __restrict__ fx,
                                                   const float* __restrict__ fy, const float* __restrict__ fz,
                                                   float om) {
  __shared__ BlkLev sb[kSmallLevelBlocks];
  const bool staged = nb <= kSmallLevelBlocks;
  pdl_trigger();
  if (staged)
    for (int q = threadIdx.x; q < nb; q += blockDim.x) sb[q] = bls[q];
  __syncthreads();
  pdl_wait();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    // info: block (bits 0-15) and the cell's wall faces (bits 16-21, W E S N B T)
    const long long gi = src[e];
    const int inf = info[e], m = inf >> 16;
    const BlkLev& B = staged ? sb[inf & 0xffff] : bls[inf & 0xffff];
    const long long sx = B.sx, sxy = B.sxy;
    float aw, ae, as, an, ab, at;
    if (VAR) {
      aw = fx[gi - 1]; ae = fx[gi]; as = fy[gi - sx]; an = fy[gi]; ab = fz[gi - sxy]; at = fz[gi];
    } else {
      const float ax = (float)B.ax, ay = (float)B.ay, az = (float)B.az;
      aw = (m & 1) ? 0.f : ax; ae = (m & 2) ? 0.f : ax;
      as = (m & 4) ? 0.f : ay; an = (m & 8) ? 0.f : ay;
      ab = (m & 16) ? 0.f : az; at = (m & 32) ? 0.f : az;
    }
    const float* P = phi + gi;
    const float sum = fmaf(at, P[sxy], fmaf(ab, P[-sxy], fmaf(an, P[sx], fmaf(as, P[-sx], fmaf(ae, P[1], aw * P[-1])))));
    phi[dst[e]] = sorf(P[0], (rhs[gi] - sum) * (1.f / -(aw + ae + as + an + ab + at)), om);
  }
}

cudaError_t launch_red_ahead(bool var, const uint32_t* dst, const uint32_t* src, const int* info, int64_t n, int nb,
                             const BlkLev* bl, float* phi, const float* rhs, const float* fx, const float* fy,
                             const float* fz, float om, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 256);
  if (var) pdl_launch(k_red_ahead<true>, g, 256, 0, st, dst, src, info, n, nb, bl, phi, rhs, fx, fy, fz, om);
  else pdl_launch(k_red_ahead<false>, g, 256, 0, st, dst, src, info, n, nb, bl, phi, rhs, fx, fy, fz, om);
  return cudaGetLastError();
}

static inline int row_grid(int nrows) {
  int g = (nrows + 7) / 8;  // 8 warps (rows) per CTA
  return g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g);
}

template <typename T>
cudaError_t launch_restrict(bool var, bool zero_phi, const BlkLev* fine, const BlkLev* coarse, RowTab rt,
                            const T* phi, const T* rhs, T* rhs_c, const T* fx, const T* fy, const T* fz,
                            cudaStream_t st) {
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = row_grid(rt.nrows);
  if (zero_phi) pdl_launch(k_restrict<T, false, true>, g, 256, 0, st, fine, coarse, rt.start, rt.nb, rt.nrows, phi, rhs, rhs_c, fx, fy, fz);
  else if (var) pdl_launch(k_restrict<T, true, false>, g, 256, 0, st, fine, coarse, rt.start, rt.nb, rt.nrows, phi, rhs, rhs_c, fx, fy, fz);
  else pdl_launch(k_restrict<T, false, false>, g, 256, 0, st, fine, coarse, rt.start, rt.nb, rt.nrows, phi, rhs, rhs_c, fx, fy, fz);
  return cudaGetLastError();
}

// mgcorr + mgbound, tiled and vectorised.  Fine rows 2k and 2k+1 (ghost
// rows 0 and ny+1 included, also through their mgbound source) interpolate
// from the same coarse rows k, k+1, and fine planes 2m, 2m+1 from the same
// coarse planes m, m+1.  So a CTA owns the plane pair (2m, 2m+1) of one
// block, a warp a row pair at a time (pairs w, w+8, ...), and a lane a group
// of VEC = 16/sizeof(T) interior cells (x0 = 1 + VEC*g, a 16-byte aligned
// address in the padded layout) of all four rows of the quad: one set of
// coarse loads (2 x 2 coarse rows, VEC/2+2 columns) serves 4 VEC fine cells;
// one vector load of the old iterate and one vector store per row.  Lanes 0
// and 1 take the ghost columns.  Same interpolation, term order and mgbound
// source as k_prolong_pairs.  Needs nx a multiple of VEC and ny, nz even.
template <typename T, bool ZERO_OLD>
__global__ void __launch_bounds__(256, 3) k_prolong_vec(const BlkLev* __restrict__ fine, const BlkLev* __restrict__ coarse,
                                                     const Tile* __restrict__ tiles, const T* __restrict__ phi_c,
                                                     const T* __restrict__ old, T* __restrict__ out) {
  pdl_trigger();
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int NC = VEC / 2 + 2;  // coarse columns a group reads
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const Tile t = tiles[blockIdx.x];
  const BlkLev F = fine[t.b];
  const BlkLev C = coarse[t.b];
  const int lane = threadIdx.x & 31;
  const int ph = F.phys;
  // the two planes of the pair and their mgbound sources
  int zq[2], szq[2];
  T wz0[2], wz1[2];
#pragma unroll
  for (int iz = 0; iz < 2; ++iz) {
    const int z = t.z0 + iz;
    int sz = z;
    if (z == 0 && (ph & 16)) sz = 1;
    if (z == F.nz + 1 && (ph & 32)) sz = F.nz;
    zq[iz] = z;
    szq[iz] = sz;
    wz0[iz] = (sz & 1) ? T(1) : T(3);
    wz1[iz] = (sz & 1) ? T(3) : T(1);
  }
  const long long cy = C.sx, cz = C.sxy;
  const int ng = F.nx / VEC;
  pdl_wait();  // everything above reads only setup data
#pragma unroll 2
  for (int k = threadIdx.x >> 5; k <= F.ny / 2; k += 8) {  // two row pairs in flight a warp
    // rows 2k, 2k+1 and their sources
    int yq[2], syq[2];
    T wy0[2], wy1[2];
#pragma unroll
    for (int iy = 0; iy < 2; ++iy) {
      const int y = 2 * k + iy;
      int sy = y;
      if (y == 0 && (ph & 4)) sy = 1;
      if (y == F.ny + 1 && (ph & 8)) sy = F.ny;
      yq[iy] = y;
      syq[iy] = sy;
      wy0[iy] = (sy & 1) ? T(1) : T(3);
      wy1[iy] = (sy & 1) ? T(3) : T(1);
    }
    // coarse row k, plane m of the quad (the same for its four rows)
    const T* Pc = phi_c + C.off + (long long)(szq[0] >> 1) * C.sxy + (long long)(syq[0] >> 1) * C.sx;
    const T* R00 = Pc;
    const T* R10 = Pc + cy;
    const T* R01 = Pc + cz;
    const T* R11 = Pc + cy + cz;
    for (int g = lane; g < ng; g += 32) {
      const int x0 = 1 + VEC * g;
      T cq[4][NC];
      const int c0 = x0 >> 1;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        cq[0][c] = R00[c0 + c];
        cq[1][c] = R10[c0 + c];
        cq[2][c] = R01[c0 + c];
        cq[3][c] = R11[c0 + c];
      }
#pragma unroll
      for (int iz = 0; iz < 2; ++iz)
#pragma unroll
        for (int iy = 0; iy < 2; ++iy) {
          const T w00 = wy0[iy] * wz0[iz], w10 = wy1[iy] * wz0[iz], w01 = wy0[iy] * wz1[iz],
                  w11 = wy1[iy] * wz1[iz];  // [dj][dk]
          // the eight weights of odd (wo) and even (we) fine columns: products of small integers
          const T wo[8] = {w00, w10, w01, w11, T(3) * w00, T(3) * w10, T(3) * w01, T(3) * w11};
          const T we[8] = {T(3) * w00, T(3) * w10, T(3) * w01, T(3) * w11, w00, w10, w01, w11};
          const long long ro = F.off + (long long)szq[iz] * F.sxy + (long long)syq[iy] * F.sx;
          V ov;
          if (ZERO_OLD) ov = V{};
          else ov = *reinterpret_cast<const V*>(old + ro + x0);
          T o[VEC], r[VEC];
          *reinterpret_cast<V*>(o) = ov;
#pragma unroll
          for (int m = 0; m < VEC; ++m) {
            const int kq = (m + 1) >> 1;  // (x >> 1) - (x0 >> 1) for x = x0 + m, x0 odd
            const T* W = (m & 1) ? we : wo;  // x0 + m odd for even m
            // term order (di,dj,dk): 000, 010, 001, 011, 100, 110, 101, 111 (mgsolver.for:838-892)
            T sum;
            if (sizeof(T) == 8) {
              sum = W[0] * cq[0][kq];
              sum = sum + W[1] * cq[1][kq];
              sum = sum + W[2] * cq[2][kq];
              sum = sum + W[3] * cq[3][kq];
              sum = sum + W[4] * cq[0][kq + 1];
              sum = sum + W[5] * cq[1][kq + 1];
              sum = sum + W[6] * cq[2][kq + 1];
              sum = sum + W[7] * cq[3][kq + 1];
              r[m] = o[m] + sum / T(64);
            } else {  // FP32 inner solve: fused multiply-adds
              sum = W[0] * cq[0][kq];
              sum = fma(W[1], cq[1][kq], sum);
              sum = fma(W[2], cq[2][kq], sum);
              sum = fma(W[3], cq[3][kq], sum);
              sum = fma(W[4], cq[0][kq + 1], sum);
              sum = fma(W[5], cq[1][kq + 1], sum);
              sum = fma(W[6], cq[2][kq + 1], sum);
              sum = fma(W[7], cq[3][kq + 1], sum);
              r[m] = fma(sum, T(1.0 / 64), o[m]);
            }
          }
          *reinterpret_cast<V*>(out + F.off + (long long)zq[iz] * F.sxy + (long long)yq[iy] * F.sx + x0) =
              *reinterpret_cast<const V*>(r);
        }
    }
    if (lane < 2) {  // ghost columns, evaluated at their mgbound source
      const int x = lane ? F.nx + 1 : 0;
      int sx = x;
      if (x == 0 && (ph & 1)) sx = 1;
      if (x == F.nx + 1 && (ph & 2)) sx = F.nx;
      const T wx0 = (sx & 1) ? T(1) : T(3), wx1 = (sx & 1) ? T(3) : T(1);
      const T* Q = Pc + (x >> 1);
#pragma unroll
      for (int iz = 0; iz < 2; ++iz)
#pragma unroll
        for (int iy = 0; iy < 2; ++iy) {
          const T w00 = wy0[iy] * wz0[iz], w10 = wy1[iy] * wz0[iz], w01 = wy0[iy] * wz1[iz],
                  w11 = wy1[iy] * wz1[iz];
          const long long ro = F.off + (long long)szq[iz] * F.sxy + (long long)syq[iy] * F.sx;
          const T o = ZERO_OLD ? T(0) : old[ro + sx];
          // term order (di,dj,dk): 000, 010, 001, 011, 100, 110, 101, 111 (mgsolver.for:838-892)
          T sum = (wx0 * w00) * Q[0];
          sum = sum + (wx0 * w10) * Q[cy];
          sum = sum + (wx0 * w01) * Q[cz];
          sum = sum + (wx0 * w11) * Q[cy + cz];
          sum = sum + (wx1 * w00) * Q[1];
          sum = sum + (wx1 * w10) * Q[1 + cy];
          sum = sum + (wx1 * w01) * Q[1 + cz];
          sum = sum + (wx1 * w11) * Q[1 + cy + cz];
          out[F.off + (long long)zq[iz] * F.sxy + (long long)yq[iy] * F.sx + x] = o + sum / T(64);
        }
    }
  }
}

template <typename T>
cudaError_t launch_prolong_vec(bool zero_old, const BlkLev* fine, const BlkLev* coarse, const Tile* tiles, int ntiles,
                               const T* phi_c, const T* old, T* out, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  if (zero_old) pdl_launch(k_prolong_vec<T, true>, ntiles, 256, 0, st, fine, coarse, tiles, phi_c, old, out);
  else pdl_launch(k_prolong_vec<T, false>, ntiles, 256, 0, st, fine, coarse, tiles, phi_c, old, out);
  return cudaGetLastError();
}
template cudaError_t launch_prolong_vec<double>(bool, const BlkLev*, const BlkLev*, const Tile*, int, const double*,
                                                const double*, double*, cudaStream_t);
template cudaError_t launch_prolong_vec<float>(bool, const BlkLev*, const BlkLev*, const Tile*, int, const float*,
                                               const float*, float*, cudaStream_t);

template <typename T>
cudaError_t launch_prolong(bool zero_old, const BlkLev* fine, const BlkLev* coarse, RowTab rt, const T* phi_c,
                           const T* old, T* out, cudaStream_t st) {
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = row_grid(rt.nrows);
  if (zero_old) pdl_launch(k_prolong_pairs<T, true>, g, 256, 0, st, fine, coarse, rt.start, rt.nb, rt.nrows, phi_c, old, out);
  else pdl_launch(k_prolong_pairs<T, false>, g, 256, 0, st, fine, coarse, rt.start, rt.nb, rt.nrows, phi_c, old, out);
  return cudaGetLastError();
}

int defect_grid(int nrows) {
  int g = (nrows + 7) / 8;
  return g < 1 ? 1 : (g > kDefectCtas ? kDefectCtas : g);
}

// The same defect, tiled and vectorised: one CTA per tile (kProlongRows
// consecutive rows of one plane, ghost rows and planes included; a warp every
// eighth row), a lane pairs of cells (x0, x0+1), x0 = 1 + 2g, with 16-byte
// loads of p and b (8-byte of e) and stores of p_next and rhs_out; the cells
// left and right of a pair are read singly, the ghost columns by lanes 0, 1.
// Same residual arithmetic as k_defect; per-CTA partial sums in a fixed order.
// Needs nx even and constant coefficients.
template <typename TE, typename TR, bool HAS_E>
__global__ void __launch_bounds__(256) k_defect_vec(const BlkLev* __restrict__ bls, const Tile* __restrict__ tiles,
                                                    int ntiles, const double* __restrict__ p,
                                                    const TE* __restrict__ e, double* __restrict__ p_next,
                                                    const double* __restrict__ bvec, TR* __restrict__ rhs_out,
                                                    double mean_b, double rscale, double* __restrict__ partials) {
  pdl_trigger();
  pdl_wait();
  using E2 = typename std::conditional<sizeof(TE) == 4, float2, double2>::type;
  using R2 = typename std::conditional<sizeof(TR) == 4, float2, double2>::type;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double rr = 0, bb = 0, rm = 0, rs = 0;
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const double rsc = rscale < 0.0 ? B.dv : rscale;  // rmax measure: |r| times the block's cell volume
  const int z = t.z0;
  for (int y = t.y0 + w; y <= min(t.y0 + kProlongRows - 1, B.ny + 1); y += 8) {
    const bool row_in = y >= 1 && y <= B.ny && z >= 1 && z <= B.nz;
    const long long rowg = B.off + (long long)z * B.sxy + (long long)y * B.sx;
    auto pv = [&](long long j) -> double {
      if (HAS_E) return p[j] + (double)e[j];
      return p[j];
    };
    auto pv2 = [&](long long j) -> double2 {  // j: 16-byte aligned pair
      double2 a = *reinterpret_cast<const double2*>(p + j);
      if (HAS_E) {
        const E2 d = *reinterpret_cast<const E2*>(e + j);
        a.x = a.x + (double)d.x;
        a.y = a.y + (double)d.y;
      }
      return a;
    };
    const int ng = B.nx >> 1;
    for (int g = lane; g < ng; g += 32) {
      const int x0 = 1 + 2 * g;
      const long long i = rowg + x0;
      const double2 pc = pv2(i);
      if (HAS_E) *reinterpret_cast<double2*>(p_next + i) = pc;
      if (!row_in) continue;
      const double2 so = pv2(i - B.sx), no = pv2(i + B.sx), bo = pv2(i - B.sxy), to = pv2(i + B.sxy);
      const double wv = pv(i - 1), ev = pv(i + 2);
      const double2 bv = *reinterpret_cast<const double2*>(bvec + i);
      const Coef<double> c0 = cell_coef<double, false>(B, x0, y, z, i - B.off, nullptr, nullptr, nullptr);
      const Coef<double> c1 = cell_coef<double, false>(B, x0 + 1, y, z, i + 1 - B.off, nullptr, nullptr, nullptr);
      const double ap0 = coef_ap(c0), ap1 = coef_ap(c1);
      const double r0 = bv.x - (c0.aw * wv + c0.ae * pc.y + c0.as * so.x + c0.an * no.x + c0.ab * bo.x +
                                c0.at * to.x + ap0 * pc.x);
      const double r1 = bv.y - (c1.aw * pc.x + c1.ae * ev + c1.as * so.y + c1.an * no.y + c1.ab * bo.y +
                                c1.at * to.y + ap1 * pc.y);
      R2 ro;
      ro.x = (TR)(r0 - mean_b);
      ro.y = (TR)(r1 - mean_b);
      *reinterpret_cast<R2*>(rhs_out + i) = ro;
      rr += r0 * r0;
      rr += r1 * r1;
      bb += bv.x * bv.x;
      bb += bv.y * bv.y;
      rm = fmax(rm, fabs(r0) * rsc);
      rm = fmax(rm, fabs(r1) * rsc);
      rs += r0;
      rs += r1;
    }
    if (HAS_E && lane < 2) {  // ghost columns: p += e only
      const long long i = rowg + (lane ? B.nx + 1 : 0);
      p_next[i] = pv(i);
    }
  }
  block_reduce4<256>(rr, bb, rm, rs, partials + 4 * (size_t)blockIdx.x);
}

// The same defect as a z march: a CTA owns kDefectRows rows of one block
// over a chunk of planes, a warp a row (plus a warp for each halo row), a
// lane GP pairs of cells (x0, x0+1), x0 = 1 + 2(lane + 32k), and the lanes
// 0 and 1 the ghost columns x = 0 and x = nx + 1.  Every thread streams its
// own cells of p, e and b into a private ring of kDefectRing planes in
// shared memory with asynchronous copies (cp.async) issued kDefectRing
// planes ahead, so DRAM sees the whole chunk in flight without registers
// held for it; a thread reads back only what it copied itself (its own
// wait_group orders it), so the ring needs no barrier.  p (+e) of planes
// z-1 .. z+1 of its own cells stays in registers; the rows y-1, y+1 and the
// cells left and right of a pair come from plane z staged in shared memory
// (two buffers, one barrier a plane).  Cells written: p_next over the whole
// padded block (ghost rows, columns and planes by the tiles and lanes that
// hold them), rhs_out and the sums over the interior.  Same residual
// arithmetic as k_defect; per-CTA partial sums in a fixed order.  Needs nx
// even, nx <= 64 GP and constant coefficients.
constexpr int kDefectRows = 8;
constexpr int kDefectRing = 3;
template <typename TE, int GP>
struct DefectCfg {
  static constexpr int R = kDefectRows + 2;  // rows with the two halo rows
  static constexpr int RW = 64 * GP + 4;     // row: [pad, x = 0 .. nx + 1, pad...]; pairs 16-byte aligned
  static constexpr size_t STAGE = 2ull * R * RW * sizeof(double);
  static constexpr size_t RAWP = (size_t)kDefectRing * R * RW * sizeof(double);
  static constexpr size_t RAWE = (size_t)kDefectRing * R * RW * sizeof(TE);
  static constexpr size_t RAWB = (size_t)kDefectRing * kDefectRows * RW * sizeof(double);
  static constexpr size_t SMEM = STAGE + RAWP + RAWE + RAWB + 128;  // + alignment of the dynamic base
  static_assert(SMEM <= 232448, "defect ring exceeds shared memory");
};

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_pair(T* sdst, const T* gsrc) {  // two elements
  if (sizeof(T) == 8) cp_async16(sdst, gsrc);
  else cp_async8(sdst, gsrc);
}
template <typename T>
__device__ __forceinline__ void cp_async_one(T* sdst, const T* gsrc) {
  if (sizeof(T) == 8) cp_async8(sdst, gsrc);
  else cp_async4(sdst, gsrc);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename TE, typename TR, bool HAS_E, int GP>
__global__ void __launch_bounds__(32 * (kDefectRows + 2)) k_defect_march(
    const BlkLev* __restrict__ bls, const Tile* __restrict__ tiles, int zc, const double* __restrict__ p,
    const TE* __restrict__ e, double* __restrict__ p_next, const double* __restrict__ bvec, TR* __restrict__ rhs_out,
    double mean_b, double rscale, double* __restrict__ partials) {
  pdl_trigger();
  using C = DefectCfg<TE, GP>;
  constexpr int R = C::R, RW = C::RW, NR = kDefectRing;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_base128(smem_raw);
  double(*sm)[R][RW] = reinterpret_cast<double(*)[R][RW]>(base);
  double(*rp)[R][RW] = reinterpret_cast<double(*)[R][RW]>(base + C::STAGE);
  TE(*re)[R][RW] = reinterpret_cast<TE(*)[R][RW]>(base + C::STAGE + C::RAWP);
  double(*rb)[kDefectRows][RW] = reinterpret_cast<double(*)[kDefectRows][RW]>(base + C::STAGE + C::RAWP + C::RAWE);
  using R2 = typename std::conditional<sizeof(TR) == 4, float2, double2>::type;
  using E2 = typename std::conditional<sizeof(TE) == 4, float2, double2>::type;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double rr = 0, bb = 0, rm = 0, rs = 0;
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bls[t.b];
  const double rsc = rscale < 0.0 ? B.dv : rscale;  // rmax measure: |r| times the block's cell volume
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long sx = B.sx, sxy = B.sxy;
  const int zs = t.z0, ze = min(t.z0 + zc - 1, nz);
  const int y = t.y0 - 1 + w;
  const bool yin = y >= 0 && y <= ny + 1;                              // the row exists (ghost rows included)
  const bool own = y >= t.y0 && y <= min(t.y0 + kDefectRows - 1, ny);  // interior rows of this tile
  const bool wr = HAS_E && (own || (yin && (y == 0 || y == ny + 1)));  // rows whose p_next this tile writes
  const long long row = B.off + (long long)y * sx;                     // cell (0, y, 0)
  const int ng = nx >> 1;
  bool gv[GP];
#pragma unroll
  for (int k = 0; k < GP; ++k) gv[k] = yin && lane + 32 * k < ng;
  auto x0 = [&](int k) { return 1 + 2 * (lane + 32 * k); };
  const bool gc = yin && lane < 2;  // lanes 0 and 1 hold the ghost columns x = 0 and x = nx + 1
  const int gx = lane == 0 ? 0 : nx + 1;

  // copy this thread's cells of plane z (p, e, and b on interior planes) into ring slot z - zs + 1 (mod NR)
  auto issue = [&](int z) {
    if (z <= ze + 1) {
      const int sl = (z - zs + 1) % NR;
      const long long rz = row + (long long)z * sxy;
#pragma unroll
      for (int k = 0; k < GP; ++k)
        if (gv[k]) {
          cp_async_pair(&rp[sl][w][1 + x0(k)], p + rz + x0(k));
          if (HAS_E) cp_async_pair(&re[sl][w][1 + x0(k)], e + rz + x0(k));
          if (own && z >= zs && z <= ze) cp_async_pair(&rb[sl][w - 1][1 + x0(k)], bvec + rz + x0(k));
        }
      if (gc) {
        cp_async_one(&rp[sl][w][1 + gx], p + rz + gx);
        if (HAS_E) cp_async_one(&re[sl][w][1 + gx], e + rz + gx);
      }
    }
    cp_async_commit();  // one group per plane, empty ones included
  };
  // this thread's p (+ e) of planes z-1, z, z+1 and b of planes z, z+1
  double2 P[3][GP], bz[GP], bz1[GP];
  double G[3];
  // plane z from its ring slot (the copies of the NR-1 later planes may still be in flight)
  auto take = [&](double2 (&q)[GP], double& g, double2 (&bq)[GP], int z) {
    cp_async_wait<NR - 1>();
    const int sl = (z - zs + 1) % NR;
#pragma unroll
    for (int k = 0; k < GP; ++k)
      if (gv[k]) {
        double2 a = *reinterpret_cast<const double2*>(&rp[sl][w][1 + x0(k)]);
        if (HAS_E) {
          const E2 d = *reinterpret_cast<const E2*>(&re[sl][w][1 + x0(k)]);
          a.x = a.x + (double)d.x;
          a.y = a.y + (double)d.y;
        }
        q[k] = a;
        if (own && z >= zs && z <= ze) bq[k] = *reinterpret_cast<const double2*>(&rb[sl][w - 1][1 + x0(k)]);
      }
    if (gc) g = HAS_E ? rp[sl][w][1 + gx] + (double)re[sl][w][1 + gx] : rp[sl][w][1 + gx];
    issue(z + NR);  // the slot is free again (this thread read back only what it copied)
  };
  auto store_next = [&](const double2 (&q)[GP], double g, int z) {  // p_next = p + e of plane z
    const long long rz = row + (long long)z * sxy;
#pragma unroll
    for (int k = 0; k < GP; ++k)
      if (gv[k]) *reinterpret_cast<double2*>(p_next + rz + x0(k)) = q[k];
    if (gc) p_next[rz + gx] = g;
  };

  pdl_wait();  // everything above reads only setup data
#pragma unroll
  for (int q = 0; q < NR; ++q) issue(zs - 1 + q);
  // face coefficients (mgsolver.for:186-205): walls zero the face term; a pair
  // (x0, x0+1) starts at an odd x, so only x0 can be the west wall cell and
  // only x0+1 the east one (nx is even)
  const double cax = B.ax, cay = B.ay, caz = B.az;
  const double cas = (y == 1 && (B.phys & 4)) ? 0.0 : cay, can = (y == ny && (B.phys & 8)) ? 0.0 : cay;
  double aw0[GP], ae1[GP];
#pragma unroll
  for (int k = 0; k < GP; ++k) {
    aw0[k] = (x0(k) == 1 && (B.phys & 1)) ? 0.0 : cax;
    ae1[k] = (x0(k) + 1 == nx && (B.phys & 2)) ? 0.0 : cax;
  }
  take(P[0], G[0], bz, zs - 1);
  take(P[1], G[1], bz, zs);
  if (wr && zs == 1) store_next(P[0], G[0], 0);  // ghost plane below
  for (int z = zs; z <= ze; ++z) {
    const double cab = (z == 1 && (B.phys & 16)) ? 0.0 : caz, cat = (z == nz && (B.phys & 32)) ? 0.0 : caz;
    const int buf = z & 1;
    const long long rz = row + (long long)z * sxy;
    take(P[2], G[2], bz1, z + 1);
    // stage plane z
    if (yin) {
#pragma unroll
      for (int k = 0; k < GP; ++k)
        if (gv[k]) *reinterpret_cast<double2*>(&sm[buf][w][1 + x0(k)]) = P[1][k];
      if (gc) sm[buf][w][1 + gx] = G[1];
    }
    __syncthreads();
    if (own) {
#pragma unroll
      for (int k = 0; k < GP; ++k) {
        if (!gv[k]) continue;
        const int xa = x0(k);
        const double2 pc = P[1][k], bo = P[0][k], to = P[2][k], b2 = bz[k];
        const double2 so = *reinterpret_cast<const double2*>(&sm[buf][w - 1][1 + xa]);
        const double2 no = *reinterpret_cast<const double2*>(&sm[buf][w + 1][1 + xa]);
        const double wv = sm[buf][w][xa], ev = sm[buf][w][xa + 3];
        const long long i = rz + xa;
        // the coefficients of cell_coef, from the thread's x and y faces and the plane's z faces
        const Coef<double> c0{aw0[k], cax, cas, can, cab, cat};
        const Coef<double> c1{cax, ae1[k], cas, can, cab, cat};
        const double ap0 = coef_ap(c0), ap1 = coef_ap(c1);
        const double r0 = b2.x - (c0.aw * wv + c0.ae * pc.y + c0.as * so.x + c0.an * no.x + c0.ab * bo.x +
                                  c0.at * to.x + ap0 * pc.x);
        const double r1 = b2.y - (c1.aw * pc.x + c1.ae * ev + c1.as * so.y + c1.an * no.y + c1.ab * bo.y +
                                  c1.at * to.y + ap1 * pc.y);
        R2 ro;
        ro.x = (TR)(r0 - mean_b);
        ro.y = (TR)(r1 - mean_b);
        *reinterpret_cast<R2*>(rhs_out + i) = ro;
        rr += r0 * r0;
        rr += r1 * r1;
        bb += b2.x * b2.x;
        bb += b2.y * b2.y;
        rm = fmax(rm, fabs(r0) * rsc);
        rm = fmax(rm, fabs(r1) * rsc);
        rs += r0;
        rs += r1;
      }
    }
    if (wr) store_next(P[1], G[1], z);
#pragma unroll
    for (int k = 0; k < GP; ++k) {
      P[0][k] = P[1][k];
      P[1][k] = P[2][k];
      bz[k] = bz1[k];
    }
    G[0] = G[1];
    G[1] = G[2];
  }
  cp_async_wait<0>();  // nothing of this CTA's copies outlives it
  if (wr && ze == nz) store_next(P[1], G[1], nz + 1);  // ghost plane above (now the middle plane)
  block_reduce4<32 * (kDefectRows + 2)>(rr, bb, rm, rs, partials + 4 * (size_t)blockIdx.x);
}

template <typename TE, int GP>
static cudaError_t defect_march_attr() {
  return cudaFuncSetAttribute(k_defect_march<TE, TE, true, GP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)DefectCfg<TE, GP>::SMEM) != cudaSuccess
             ? cudaGetLastError()
             : cudaFuncSetAttribute(k_defect_march<TE, TE, false, GP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)DefectCfg<TE, GP>::SMEM);
}
cudaError_t defect_march_attributes() {
  cudaError_t e;
  if ((e = defect_march_attr<float, 1>()) || (e = defect_march_attr<float, 2>()) || (e = defect_march_attr<float, 4>()) ||
      (e = defect_march_attr<double, 1>()) || (e = defect_march_attr<double, 2>()) ||
      (e = defect_march_attr<double, 4>()))
    return e;
  return cudaSuccess;
}

template <typename TE, typename TR>
cudaError_t launch_defect_march(int gp, const BlkLev* bl, const Tile* tiles, int ntiles, int zc, const double* p,
                                const TE* e, double* p_next, const double* b, TR* rhs_out, double mean_b,
                                double rscale, double* partials, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  constexpr int NT = 32 * (kDefectRows + 2);
#define H3D_DM(G)                                                                                                    \
  if (gp == G) {                                                                                                     \
    constexpr size_t SM = DefectCfg<TE, G>::SMEM;                                                                    \
    if (e) pdl_launch(k_defect_march<TE, TR, true, G>, ntiles, NT, SM, st, bl, tiles, zc, p, e, p_next, b, rhs_out, \
                      mean_b, rscale, partials);                                                                     \
    else pdl_launch(k_defect_march<TE, TR, false, G>, ntiles, NT, SM, st, bl, tiles, zc, p, e, p_next, b, rhs_out,  \
                    mean_b, rscale, partials);                                                                       \
    return cudaGetLastError();                                                                                       \
  }
  H3D_DM(1)
  H3D_DM(2)
  H3D_DM(4)
#undef H3D_DM
  return cudaErrorInvalidValue;
}
template cudaError_t launch_defect_march<double, double>(int, const BlkLev*, const Tile*, int, int, const double*,
                                                         const double*, double*, const double*, double*, double,
                                                         double, double*, cudaStream_t);
template cudaError_t launch_defect_march<float, float>(int, const BlkLev*, const Tile*, int, int, const double*,
                                                       const float*, double*, const double*, float*, double, double,
                                                       double*, cudaStream_t);
int defect_march_rows() { return kDefectRows; }

template <typename TE, typename TR>
cudaError_t launch_defect_vec(const BlkLev* bl, const Tile* tiles, int ntiles, const double* p, const TE* e,
                              double* p_next, const double* b, TR* rhs_out, double mean_b, double rscale,
                              double* partials, int grid, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  grid = ntiles;  // one tile per CTA (partials holds one quadruple per tile)
  if (e) pdl_launch(k_defect_vec<TE, TR, true>, grid, 256, 0, st, bl, tiles, ntiles, p, e, p_next, b, rhs_out, mean_b, rscale, partials);
  else pdl_launch(k_defect_vec<TE, TR, false>, grid, 256, 0, st, bl, tiles, ntiles, p, e, p_next, b, rhs_out, mean_b, rscale, partials);
  return cudaGetLastError();
}
template cudaError_t launch_defect_vec<double, double>(const BlkLev*, const Tile*, int, const double*, const double*,
                                                       double*, const double*, double*, double, double, double*, int,
                                                       cudaStream_t);
template cudaError_t launch_defect_vec<float, float>(const BlkLev*, const Tile*, int, const double*, const float*,
                                                     double*, const double*, float*, double, double, double*, int,
                                                     cudaStream_t);

template <typename TE, typename TR>
cudaError_t launch_defect(bool var, const BlkLev* bl, RowTab rt, const double* p, const TE* e, double* p_next,
                          const double* b, TR* rhs_out, double mean_b, double rscale, const double* fx,
                          const double* fy, const double* fz, double* partials, cudaStream_t st) {
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = defect_grid(rt.nrows);
  if (e) {
    if (var) pdl_launch(k_defect<TE, TR, true, true>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, p, e, p_next, b, rhs_out, mean_b, rscale, fx, fy, fz, partials);
    else pdl_launch(k_defect<TE, TR, true, false>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, p, e, p_next, b, rhs_out, mean_b, rscale, fx, fy, fz, partials);
  } else {
    if (var) pdl_launch(k_defect<TE, TR, false, true>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, p, e, p_next, b, rhs_out, mean_b, rscale, fx, fy, fz, partials);
    else pdl_launch(k_defect<TE, TR, false, false>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, p, e, p_next, b, rhs_out, mean_b, rscale, fx, fy, fz, partials);
  }
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// TMA-staged restriction (mgrestr, mgsolver.for:623-766): fine residuals
// summed into the coarse right-hand side, with the arithmetic of
// k_restrict_tile (same residual operand order, same child order: i fastest,
// then j, then k), so FP64 stays bit-exact.  A CTA owns TYC coarse rows of a
// block (whole rows) and a range of coarse planes; fine planes arrive by TMA
// (iterate: fine rows 2Y0-2 .. 2Y0+2TYC-1, right-hand side: rows 2Y0-1 ..
// 2Y0+2TYC-2) into an NS-slot ring, D planes ahead, one barrier per fine
// plane.  Thread (tr, tc) owns coarse cells X = 1 + tc + k*TPR of coarse row
// Y0 + tr and reads each pair of fine children (x = 2X-1, 2X) with one
// 8- (FP32) or 16-byte (FP64) shared-memory load.
template <typename T, int TPR, int CPX, int TYC, int NS>
struct RTmaCfg {
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int SPMAX = ((2 * CPX * TPR + 2 + kXOff + VEC - 1) / VEC) * VEC;
  static constexpr int PSLOT = ((SPMAX * (2 * TYC + 2) * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int RSLOT = ((SPMAX * (2 * TYC) * (int)sizeof(T) + 127) / 128) * 128;
  static constexpr int SLOT = PSLOT + RSLOT;
  static constexpr size_t SMEM = (size_t)NS * SLOT + 128 + NS * 8;
  static_assert(SMEM <= 232448, "ring exceeds shared memory");
};

template <typename T>
struct Pair {
  T x, y;
};

template <typename T, int TPR, int CPX, int TYC, int NS, int D, bool VAR, bool ZERO>
__global__ void __launch_bounds__(TPR* TYC) k_restrict_tma(const BlkLev* __restrict__ fine,
                                                          const BlkLev* __restrict__ coarse,
                                                          const Tile* __restrict__ tiles, int zc,
                                                          const CUtensorMap* __restrict__ pmaps,
                                                          const CUtensorMap* __restrict__ rmaps,
                                                          T* __restrict__ rhs_c, const T* __restrict__ fx,
                                                          const T* __restrict__ fy, const T* __restrict__ fz,
                                                          int* err) {
  pdl_trigger();
  using C = RTmaCfg<T, TPR, CPX, TYC, NS>;
  static_assert(D + 2 <= NS, "a fine plane is read until the phase after its own");
  using P2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_base128(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NS * C::SLOT);

  const Tile t = tiles[blockIdx.x];
  const BlkLev F = fine[t.b];
  const BlkLev Cc = coarse[t.b];
  const CUtensorMap* pmap = pmaps + t.b;
  const CUtensorMap* rmap = rmaps + t.b;
  const T* FX = VAR ? fx + F.off : nullptr;
  const T* FY = VAR ? fy + F.off : nullptr;
  const T* FZ = VAR ? fz + F.off : nullptr;
  const int Y0 = t.y0, Z0 = t.z0;
  const int Z1 = min(Z0 + zc - 1, Cc.nz);
  const int zfa = 2 * Z0 - 1, zfb = 2 * Z1;  // fine planes of the chunk
  const int BX = ((F.nx + 2 + kXOff + C::VEC - 1) / C::VEC) * C::VEC;
  const uint32_t pbytes = ZERO ? 0u : (uint32_t)(BX * (2 * TYC + 2) * (int)sizeof(T));
  const uint32_t tx_bytes = pbytes + (uint32_t)(BX * 2 * TYC * (int)sizeof(T));
  const int tr = threadIdx.x / TPR, tc = threadIdx.x - (threadIdx.x / TPR) * TPR;
  const int Y = Y0 + tr;
  const bool yok = Y <= Cc.ny;
  const bool leader = threadIdx.x == 0;
  bool bad = false;

  if (leader) {
    for (int q = 0; q < NS; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + q)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  pdl_wait();  // everything above reads only setup data

  auto pslot = [&](int q) -> const T* { return reinterpret_cast<const T*>(base + (q % NS) * C::SLOT); };
  auto rslot = [&](int q) -> const T* { return reinterpret_cast<const T*>(base + (q % NS) * C::SLOT + C::PSLOT); };
  int last_q = -1;  // last plane issued (leader)
  auto issue = [&](int q) {  // leader only
    last_q = q;
    const uint32_t bar = smem_u32(bars + q % NS);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    if (!ZERO)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
              "r"(smem_u32(pslot(q))),
          "l"(reinterpret_cast<uint64_t>(pmap)), "r"(0), "r"(2 * Y0 - 2), "r"(q), "r"(bar)
          : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(rslot(q))),
        "l"(reinterpret_cast<uint64_t>(rmap)), "r"(0), "r"(2 * Y0 - 1), "r"(q), "r"(bar)
        : "memory");
  };
  auto wait_plane = [&](int q) {
    const uint32_t parity = (uint32_t)(((q - zfa + 1) / NS) & 1);
    mbar_wait(smem_u32(bars + q % NS), parity, err, bad);
  };

  T sum[CPX];
#pragma unroll
  for (int k = 0; k < CPX; ++k) sum[k] = T(0);
  if (leader)
    for (int q = zfa - 1; q <= min(zfa + D, zfb + 1); ++q) issue(q);
  wait_plane(zfa - 1);
  wait_plane(zfa);
  for (int zf = zfa; zf <= zfb; ++zf) {
    wait_plane(zf + 1);
    if (yok) {
      const T* S = pslot(zf);
      const T* Sm = pslot(zf - 1);
      const T* Sp = pslot(zf + 1);
      const T* R = rslot(zf);
#pragma unroll
      for (int k = 0; k < CPX; ++k) {
        const int X = 1 + tc + k * TPR;
        if (X > Cc.nx) continue;
        const int ca = 2 * X - 1 + kXOff;  // smem column of the first child (even: aligned pair)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
          const int y = 2 * Y - 1 + dj;
          const int ro = (2 * tr + 1 + dj) * BX + ca;  // iterate slot offset of the pair
          const P2 rh = *reinterpret_cast<const P2*>(R + (2 * tr + dj) * BX + ca);
          T ra, rb;
          if (ZERO) {
            ra = rh.x - T(0);
            rb = rh.y - T(0);
          } else {
            const P2 cen = *reinterpret_cast<const P2*>(S + ro);
            const P2 up = *reinterpret_cast<const P2*>(S + ro - BX);
            const P2 dn = *reinterpret_cast<const P2*>(S + ro + BX);
            const P2 bo = *reinterpret_cast<const P2*>(Sm + ro);
            const P2 to = *reinterpret_cast<const P2*>(Sp + ro);
            const T wa = S[ro - 1], eb = S[ro + 2];
            const int xa = 2 * X - 1;
            const long long ia = (long long)zf * F.sxy + (long long)y * F.sx + xa;
            const Coef<T> c0 = cell_coef<T, VAR>(F, xa, y, zf, ia, FX, FY, FZ);
            const Coef<T> c1 = cell_coef<T, VAR>(F, xa + 1, y, zf, ia + 1, FX, FY, FZ);
            const T ap0 = coef_ap(c0), ap1 = coef_ap(c1);
            ra = rh.x - (c0.aw * wa + c0.ae * cen.y + c0.as * up.x + c0.an * dn.x + c0.ab * bo.x + c0.at * to.x +
                         ap0 * cen.x);
            rb = rh.y - (c1.aw * cen.x + c1.ae * eb + c1.as * up.y + c1.an * dn.y + c1.ab * bo.y + c1.at * to.y +
                         ap1 * cen.y);
          }
          sum[k] = ((zf & 1) && dj == 0) ? ra : sum[k] + ra;
          sum[k] = sum[k] + rb;
        }
        if (!(zf & 1))
          rhs_c[Cc.off + (long long)(zf >> 1) * Cc.sxy + (long long)Y * Cc.sx + X] = T(0.125) * sum[k];
      }
    }
    __syncthreads();
    if (leader && !bad && zf + D + 1 <= zfb + 1) issue(zf + D + 1);
  }
  if (leader && bad) drain_ring(bars, NS, zfa - 1, last_q, err);
}

// ---- tile restriction ------------------------------------------------------
// 0-3 plain-load tiles (k_restrict_tile); 4+ TMA-staged (k_restrict_tma)
static const RestrictShape kRShapes[] = {{16, 1, 8, 0}, {32, 1, 8, 0}, {32, 2, 4, 0}, {32, 4, 4, 0},
                                          {32, 2, 4, 1},  {32, 2, 8, 1}, {16, 2, 8, 1}, {32, 1, 8, 1},
                                          {16, 1, 8, 1},  {32, 4, 4, 1}, {64, 1, 4, 1}};
int rtma_tyc_index(int tyc) { return tyc == 4 ? 0 : tyc == 8 ? 1 : -1; }
int num_restrict_shapes() { return (int)(sizeof(kRShapes) / sizeof(kRShapes[0])); }
RestrictShape restrict_shape(int v) { return kRShapes[v]; }

template <typename T, int TPR, int CPX, int TYC>
static constexpr size_t rtile_smem() {
  return 3 * (size_t)(2 * TYC + 2) * (size_t)(2 * CPX * TPR + 4) * sizeof(T);
}

template <typename T, int TPR, int CPX, int TYC>
static cudaError_t rtile_attr() {
  const int sm = (int)rtile_smem<T, TPR, CPX, TYC>();
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_restrict_tile<T, true, false, TPR, CPX, TYC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  if ((e = cudaFuncSetAttribute(k_restrict_tile<T, false, false, TPR, CPX, TYC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  return cudaFuncSetAttribute(k_restrict_tile<T, false, true, TPR, CPX, TYC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

template <typename T, int TPR, int CPX, int TYC>
static cudaError_t rtile_dispatch(bool var, bool zero, const BlkLev* fine, const BlkLev* coarse, const Tile* tiles,
                                  int ntiles, int zc, const T* phi, const T* rhs, T* rhs_c, const T* fx, const T* fy,
                                  const T* fz, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  constexpr size_t SM = rtile_smem<T, TPR, CPX, TYC>();
  if (zero) pdl_launch(k_restrict_tile<T, false, true, TPR, CPX, TYC>, ntiles, TPR * TYC, SM, st, fine, coarse, tiles, zc, phi, rhs, rhs_c, fx, fy, fz);
  else if (var) pdl_launch(k_restrict_tile<T, true, false, TPR, CPX, TYC>, ntiles, TPR * TYC, SM, st, fine, coarse, tiles, zc, phi, rhs, rhs_c, fx, fy, fz);
  else pdl_launch(k_restrict_tile<T, false, false, TPR, CPX, TYC>, ntiles, TPR * TYC, SM, st, fine, coarse, tiles, zc, phi, rhs, rhs_c, fx, fy, fz);
  return cudaGetLastError();
}

#define H3D_RSHAPES(X) X(0, 16, 1, 8) X(1, 32, 1, 8) X(2, 32, 2, 4) X(3, 32, 4, 4)

template <typename T, int TPR, int CPX, int TYC>
static constexpr int rtma_ns() {
  return RTmaCfg<T, TPR, CPX, TYC, 5>::SMEM <= 232448 / 2 ? 5 : 4;
}

template <typename T, int TPR, int CPX, int TYC>
static cudaError_t rtma_attr() {
  constexpr int NS = rtma_ns<T, TPR, CPX, TYC>();
  const int sm = (int)RTmaCfg<T, TPR, CPX, TYC, NS>::SMEM;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_restrict_tma<T, TPR, CPX, TYC, NS, NS - 2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  if ((e = cudaFuncSetAttribute(k_restrict_tma<T, TPR, CPX, TYC, NS, NS - 2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  if ((e = cudaFuncSetAttribute(k_restrict_tma<T, TPR, CPX, TYC, NS, NS - 2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
  return cudaFuncSetAttribute(k_restrict_tma<T, TPR, CPX, TYC, NS, NS - 2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

template <typename T, int TPR, int CPX, int TYC>
static cudaError_t rtma_dispatch(bool var, bool zero, const BlkLev* fine, const BlkLev* coarse, const Tile* tiles,
                                 int ntiles, int zc, const CUtensorMap* pmaps, const CUtensorMap* rmaps, T* rhs_c,
                                 const T* fx, const T* fy, const T* fz, int* err, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  constexpr int NS = rtma_ns<T, TPR, CPX, TYC>();
  constexpr int D = NS - 2;
  constexpr size_t SM = RTmaCfg<T, TPR, CPX, TYC, NS>::SMEM;
  constexpr int NT = TPR * TYC;
  if (var) {
    if (zero) pdl_launch(k_restrict_tma<T, TPR, CPX, TYC, NS, D, true, true>, ntiles, NT, SM, st, fine, coarse, tiles, zc, pmaps, rmaps, rhs_c, fx, fy, fz, err);
    else pdl_launch(k_restrict_tma<T, TPR, CPX, TYC, NS, D, true, false>, ntiles, NT, SM, st, fine, coarse, tiles, zc, pmaps, rmaps, rhs_c, fx, fy, fz, err);
  } else {
    if (zero) pdl_launch(k_restrict_tma<T, TPR, CPX, TYC, NS, D, false, true>, ntiles, NT, SM, st, fine, coarse, tiles, zc, pmaps, rmaps, rhs_c, fx, fy, fz, err);
    else pdl_launch(k_restrict_tma<T, TPR, CPX, TYC, NS, D, false, false>, ntiles, NT, SM, st, fine, coarse, tiles, zc, pmaps, rmaps, rhs_c, fx, fy, fz, err);
  }
  return cudaGetLastError();
}

#define H3D_RTMA_SHAPES(X) \
  X(4, 32, 2, 4) X(5, 32, 2, 8) X(6, 16, 2, 8) X(7, 32, 1, 8) X(8, 16, 1, 8) X(9, 32, 4, 4) X(10, 64, 1, 4)

template <typename T>
cudaError_t launch_restrict_tile(int variant, bool var, bool zero_phi, const BlkLev* fine, const BlkLev* coarse,
                                 const Tile* tiles, int ntiles, int zc, const T* phi, const T* rhs, T* rhs_c,
                                 const T* fx, const T* fy, const T* fz, const CUtensorMap* pmaps,
                                 const CUtensorMap* rmaps, int* err, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  switch (variant) {
#define X(v, tpr, cpx, tyc) \
    case v: return rtile_dispatch<T, tpr, cpx, tyc>(var, zero_phi, fine, coarse, tiles, ntiles, zc, phi, rhs, rhs_c, fx, fy, fz, st);
    H3D_RSHAPES(X)
#undef X
#define X(v, tpr, cpx, tyc)                                                                                   \
    case v:                                                                                                   \
      if (!rmaps || (!pmaps && !zero_phi)) return cudaErrorInvalidValue;                                     \
      return rtma_dispatch<T, tpr, cpx, tyc>(var, zero_phi, fine, coarse, tiles, ntiles, zc, pmaps, rmaps, rhs_c, fx, fy, fz, err, st);
    H3D_RTMA_SHAPES(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}



cudaError_t init_kernel_attributes_2() {
  cudaError_t e = cudaSuccess;
#define X(v, tpr, cpx, tyc)                                                    \
  if ((e = rtile_attr<float, tpr, cpx, tyc>()) != cudaSuccess) return e;       \
  if ((e = rtile_attr<double, tpr, cpx, tyc>()) != cudaSuccess) return e;
  H3D_RSHAPES(X)
#undef X
#define X(v, tpr, cpx, tyc)                                                   \
  if ((e = rtma_attr<float, tpr, cpx, tyc>()) != cudaSuccess) return e;       \
  if ((e = rtma_attr<double, tpr, cpx, tyc>()) != cudaSuccess) return e;
  H3D_RTMA_SHAPES(X)
#undef X
  return e;
}

template cudaError_t launch_restrict_tile<double>(int, bool, bool, const BlkLev*, const BlkLev*, const Tile*, int, int,
    const double*, const double*, double*, const double*, const double*, const double*, const CUtensorMap*, const CUtensorMap*, int*,
    cudaStream_t);
template cudaError_t launch_restrict_tile<float>(int, bool, bool, const BlkLev*, const BlkLev*, const Tile*, int, int,
    const float*, const float*, float*, const float*, const float*, const float*, const CUtensorMap*, const CUtensorMap*, int*,
    cudaStream_t);


// ---------------------------------------------------------------------------
// Host-field staging: a host block array (Fortran dims tx, ty, tz with pl
// ghost layers, x fastest) is copied whole and contiguously between host and
// a device staging buffer; these kernels move the region g0 .. (extent) of
// the canonical block (ghost layer included when g0 = 0) between staging and
// the padded device layout.
__global__ void k_stage_scatter(const double* __restrict__ stg, int tx, int ty, int pl, int g0, int ex, int ey,
                                int ez, double* __restrict__ dev, int sx, long long sxy) {
  pdl_trigger();
  pdl_wait();
  const long long n = (long long)ex * ey * ez;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % ex), y = (int)((e / ex) % ey), z = (int)(e / ((long long)ex * ey));
    const int hx = pl - 1 + g0 + x, hy = pl - 1 + g0 + y, hz = pl - 1 + g0 + z;
    dev[(long long)(g0 + z) * sxy + (long long)(g0 + y) * sx + g0 + x] = stg[((long long)hz * ty + hy) * tx + hx];
  }
}

__global__ void k_stage_gather(double* __restrict__ stg, int tx, int ty, int pl, int g0, int ex, int ey, int ez,
                               const double* __restrict__ dev, int sx, long long sxy) {
  pdl_trigger();
  pdl_wait();
  const long long n = (long long)ex * ey * ez;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % ex), y = (int)((e / ex) % ey), z = (int)(e / ((long long)ex * ey));
    const int hx = pl - 1 + g0 + x, hy = pl - 1 + g0 + y, hz = pl - 1 + g0 + z;
    stg[((long long)hz * ty + hy) * tx + hx] = dev[(long long)(g0 + z) * sxy + (long long)(g0 + y) * sx + g0 + x];
  }
}

cudaError_t launch_stage(bool to_device, double* stg, int tx, int ty, int pl, int g0, int ex, int ey, int ez,
                         double* dev, int sx, long long sxy, cudaStream_t st) {
  const long long n = (long long)ex * ey * ez;
  if (n <= 0) return cudaSuccess;
  const int grid = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (to_device) pdl_launch(k_stage_scatter, grid, 256, 0, st, stg, tx, ty, pl, g0, ex, ey, ez, dev, sx, sxy);
  else pdl_launch(k_stage_gather, grid, 256, 0, st, stg, tx, ty, pl, g0, ex, ey, ez, dev, sx, sxy);
  return cudaGetLastError();
}

cudaError_t launch_reduce4_blocks(const double* partials, const int* start, int nb, double* out, cudaStream_t st) {
  pdl_launch(k_reduce4_blocks, nb, 256, 0, st, partials, start, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce4(const double* partials, int n, double* out, cudaStream_t st) {
  pdl_launch(k_reduce4, 1, 1024, 0, st, partials, n, out);
  return cudaGetLastError();
}

cudaError_t launch_sum_interior(const BlkLev* bl, RowTab rt, const double* a, double* partials, int* nparts,
                                cudaStream_t st) {
  *nparts = 0;
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = defect_grid(rt.nrows);
  pdl_launch(k_sum_interior, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, a, partials);
  *nparts = g;
  return cudaGetLastError();
}

cudaError_t launch_shift(double* a, int64_t n, const double* s, double scale, cudaStream_t st) {
  pdl_launch(k_shift, grid_for(n, 256), 256, 0, st, a, n, s, scale);
  return cudaGetLastError();
}

cudaError_t launch_convert_d2f(const double* a, float* b, int64_t n, cudaStream_t st) {
  pdl_launch(k_d2f, grid_for(n, 256), 256, 0, st, a, b, n);
  return cudaGetLastError();
}
cudaError_t launch_convert_f2d(const float* a, double* b, int64_t n, cudaStream_t st) {
  pdl_launch(k_f2d, grid_for(n, 256), 256, 0, st, a, b, n);
  return cudaGetLastError();
}

namespace {

// ---------------------------------------------------------------------------
// Face-sum coarse coefficients (L_LSM, coarse_op = 1; not a reference
// routine).  The coefficient of a coarse face is the sum of the four fine
// face coefficients that tile it, times 1/16: 1/2 for the two half cells in
// series along the face normal (the conductance of the coarse face in the
// finite-volume form) and 1/8 for the 8-cell average the restriction makes
// of the residual (mgsolver.for:748-752), which leaves the rhs on the fine
// cell-volume scale.  With a uniform density it equals 4^-(g-1) times the
// reference's fine-spacing coefficient; across a 1000:1 density jump it keeps
// the conductance of every light-fluid path, which averaging the density
// (mgsolver.for:78-105) does not.  Sum order fixed: ((f00 + f10) + f01) + f11.
__global__ void __launch_bounds__(256) k_face_coef_sum(const BlkLev* __restrict__ fine,
                                                       const BlkLev* __restrict__ coarse,
                                                       const int* __restrict__ cta_start, int nb,
                                                       const double* __restrict__ ffx, const double* __restrict__ ffy,
                                                       const double* __restrict__ ffz, double* __restrict__ cfx,
                                                       double* __restrict__ cfy, double* __restrict__ cfz) {
  pdl_trigger();
  pdl_wait();
  const int b = find_block(cta_start, nb, blockIdx.x);
  const BlkLev C = coarse[b];
  const BlkLev F = fine[b];
  const int local = (blockIdx.x - cta_start[b]) * blockDim.x + threadIdx.x;
  const int mx = C.nx + 2, my = C.ny + 2, mz = C.nz + 2;
  if (local >= mx * my * mz) return;
  const int x = local % mx, y = (local / mx) % my, z = local / (mx * my);
  const long long ic = C.off + (long long)z * C.sxy + (long long)y * C.sx + x;
  const bool iny = y >= 1 && y <= C.ny, inz = z >= 1 && z <= C.nz, inx = x >= 1 && x <= C.nx;
  auto fi = [&](int fx_, int fy_, int fz_) { return F.off + (long long)fz_ * F.sxy + (long long)fy_ * F.sx + fx_; };
  if (x <= C.nx && iny && inz) {  // coarse face X = fine face 2X, fine rows 2Y-1..2Y, planes 2Z-1..2Z
    const int X = 2 * x, Y = 2 * y - 1, Z = 2 * z - 1;
    cfx[ic] = (((ffx[fi(X, Y, Z)] + ffx[fi(X, Y + 1, Z)]) + ffx[fi(X, Y, Z + 1)]) + ffx[fi(X, Y + 1, Z + 1)]) * 0.0625;
  }
  if (y <= C.ny && inx && inz) {
    const int X = 2 * x - 1, Y = 2 * y, Z = 2 * z - 1;
    cfy[ic] = (((ffy[fi(X, Y, Z)] + ffy[fi(X + 1, Y, Z)]) + ffy[fi(X, Y, Z + 1)]) + ffy[fi(X + 1, Y, Z + 1)]) * 0.0625;
  }
  if (z <= C.nz && inx && iny) {
    const int X = 2 * x - 1, Y = 2 * y - 1, Z = 2 * z;
    cfz[ic] = (((ffz[fi(X, Y, Z)] + ffz[fi(X + 1, Y, Z)]) + ffz[fi(X, Y + 1, Z)]) + ffz[fi(X + 1, Y + 1, Z)]) * 0.0625;
  }
}

// ---------------------------------------------------------------------------
// The projection (press.for:2-144).  Face velocities live in the level-1
// layout of the cell they belong to: u at (x,y,z) is the east face of cell
// (x,y,z) (u(i) of the reference, i = x + isp - 1), x = 0 the block's west
// face; v north faces, w top faces.

// calvel (press.for:77-144): u = ustar - dt*alfapr*(p(i+1)-p(i))/dx on the
// faces the reference updates (x = 1..nx, or 1..nx-1 when the east face is a
// physical wall: ieu = iep - 1, localparameters.for:186-192; v and w alike),
// divided by the face density 0.5*(dens(i)+dens(i+1)) for L_LSM.  Operand
// order as written there (dtal = dt*alfapr, then *(dp), /dx, /face density).
// One warp per interior row.
template <bool LSM>
__global__ void __launch_bounds__(256) k_calvel(const BlkLev* __restrict__ bls, const int* __restrict__ row_start,
                                                int nb, int nrows, const double* __restrict__ h3,
                                                const double* __restrict__ p, const double* __restrict__ dens,
                                                const double* __restrict__ us, const double* __restrict__ vs,
                                                const double* __restrict__ ws, double* __restrict__ u,
                                                double* __restrict__ v, double* __restrict__ w, double dtal) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef ref = row_of(bls, row_start, nb, rid, true);
    const BlkLev B = bls[ref.b];
    const int y = ref.y, z = ref.z;
    const double dx = h3[3 * ref.b], dy = h3[3 * ref.b + 1], dz = h3[3 * ref.b + 2];
    const int nxu = B.nx - ((B.phys & 2) ? 1 : 0);
    const bool vrow = y <= B.ny - ((B.phys & 8) ? 1 : 0);
    const bool wrow = z <= B.nz - ((B.phys & 32) ? 1 : 0);
    const long long rowg = B.off + (long long)z * B.sxy + (long long)y * B.sx;
    for (int x = 1 + lane; x <= B.nx; x += 32) {
      const long long i = rowg + x;
      const double pc = p[i];
      if (x <= nxu) {
        double t = dtal * (p[i + 1] - pc) / dx;
        if (LSM) t = t / (0.5 * (dens[i] + dens[i + 1]));
        u[i] = us[i] - t;
      }
      if (vrow) {
        double t = dtal * (p[i + B.sx] - pc) / dy;
        if (LSM) t = t / (0.5 * (dens[i] + dens[i + B.sx]));
        v[i] = vs[i] - t;
      }
      if (wrow) {
        double t = dtal * (p[i + B.sxy] - pc) / dz;
        if (LSM) t = t / (0.5 * (dens[i] + dens[i + B.sxy]));
        w[i] = ws[i] - t;
      }
    }
  }
}

// exchange(1..3) after calvel: one gather table (face ghosts of the interior
// rows, physical walls excluded) applied to the three components.
__global__ void __launch_bounds__(256) k_gather3(const uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                                 int64_t n, double* __restrict__ a0, double* __restrict__ a1,
                                                 double* __restrict__ a2) {
  pdl_trigger();
  pdl_wait();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t d = dst[e], s = src[e];
    a0[d] = a0[s];
    a1[d] = a1[s];
    a2[d] = a2[s];
  }
}

// calmas (press.for:40-62): fact = (u(i)-u(i-1))/dx + (v(j)-v(j-1))/dy +
// (w(k)-w(k-1))/dz; su = fact/dt, or sup = fact*dx*dy*dz/dt for L_LSM;
// rmax = max |fact*dx*dy*dz|.  su goes to bout (FP64) and to the level-1
// right-hand side rhs_out (as TR); per-CTA partials {sum su^2, 0, rmax,
// sum su}.
template <bool LSM, typename TR>
__global__ void __launch_bounds__(256) k_calmas(const BlkLev* __restrict__ bls, const int* __restrict__ row_start,
                                                int nb, int nrows, const double* __restrict__ h3,
                                                const double* __restrict__ u, const double* __restrict__ v,
                                                const double* __restrict__ w, double dt, double* __restrict__ bout,
                                                TR* __restrict__ rhs_out, double* __restrict__ partials) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  double ss = 0, rm = 0, rs = 0;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef ref = row_of(bls, row_start, nb, rid, true);
    const BlkLev B = bls[ref.b];
    const double dx = h3[3 * ref.b], dy = h3[3 * ref.b + 1], dz = h3[3 * ref.b + 2];
    const long long rowg = B.off + (long long)ref.z * B.sxy + (long long)ref.y * B.sx;
    for (int x = 1 + lane; x <= B.nx; x += 32) {
      const long long i = rowg + x;
      const double fact = (u[i] - u[i - 1]) / dx + (v[i] - v[i - B.sx]) / dy + (w[i] - w[i - B.sxy]) / dz;
      const double s = LSM ? fact * dx * dy * dz / dt : fact / dt;
      bout[i] = s;
      rhs_out[i] = (TR)s;
      ss += s * s;
      rs += s;
      const double a = fabs(fact * dx * dy * dz);
      if (!(a <= rm)) rm = a;  // keeps a NaN
    }
  }
  block_reduce4<256>(ss, 0.0, rm, rs, partials + 4 * (size_t)blockIdx.x);
}

// p = p + (pp - ppref) over the block and its ghost layer (newsolv_mg.for:
// 39-49, ppref = 0): one warp per row of every row.
template <typename TE>
__global__ void __launch_bounds__(256) k_padd(const BlkLev* __restrict__ bls, const int* __restrict__ row_start,
                                              int nb, int nrows, double* __restrict__ p, const TE* __restrict__ e) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  for (int rid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rid < nrows; rid += (gridDim.x * blockDim.x) >> 5) {
    const RowRef ref = row_of(bls, row_start, nb, rid, false);
    const BlkLev B = bls[ref.b];
    const long long rowg = B.off + (long long)ref.z * B.sxy + (long long)ref.y * B.sx;
    for (int x = lane; x <= B.nx + 1; x += 32) {
      const long long i = rowg + x;
      p[i] = p[i] + ((double)e[i] - 0.0);
    }
  }
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Stone's strongly implicit procedure (sipsol.for:2-205, ifi = 44), the
// reference's alternative pressure solver, on the level-1 layout with the
// constant coefficients pressure_1sweep builds (press.for:407-438: the same
// values as coeff's level 1).  The LU factors and both substitutions are
// recurrences over the predecessors (x-1, y-1, z-1) (successors for the
// backward pass), so hyperplanes x+y+z = const are the wavefronts: one CTA
// per block sweeps them in order with a CTA barrier between, every value the
// one the reference's k, i, j loops compute, in its operand order.  Factor
// and residual arrays are zero outside the interior (never written there),
// as the reference's are.
struct SipLU {
  double *lb, *lw, *ls, *lpr, *un, *ue, *ut, *res;
};

// Calls f(x, y, z, i) for every interior cell of hyperplane x+y+z = d + 3,
// spread over the CTA's threads.
template <typename F>
__device__ __forceinline__ void sip_plane(const BlkLev& B, int d, F&& f) {
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const int zmin = max(0, d - (nx - 1) - (ny - 1)), zmax = min(nz - 1, d);
  const int nzr = zmax - zmin + 1;
  for (int q = threadIdx.x; q < nzr * ny; q += blockDim.x) {
    const int z = zmin + q / ny + 1, y = q % ny + 1;
    const int x = d - (y - 1) - (z - 1) + 1;
    if (x < 1 || x > nx) continue;
    f(x, y, z, (long long)z * B.sxy + (long long)y * B.sx + x);
  }
}

__global__ void __launch_bounds__(512) k_sip_factor(const BlkLev* __restrict__ bls, SipLU lu) {
  pdl_trigger();
  pdl_wait();
  const BlkLev B = bls[blockIdx.x];
  const double alfa = 0.92, small = 1e-20;  // sipsol.for:32-33
  double *lb = lu.lb + B.off, *lw = lu.lw + B.off, *ls = lu.ls + B.off, *lpr = lu.lpr + B.off;
  double *un = lu.un + B.off, *ue = lu.ue + B.off, *ut = lu.ut + B.off;
  const long long sj = B.sx, sk = B.sxy;
  for (int d = 0; d <= (B.nx - 1) + (B.ny - 1) + (B.nz - 1); ++d) {  // sipsol.for:77-105
    sip_plane(B, d, [&](int x, int y, int z, long long q) {
      const Coef<double> c = cell_coef<double, false>(B, x, y, z, q, nullptr, nullptr, nullptr);
      const double ap = coef_ap(c);
      lb[q] = c.ab / (1. + alfa * (un[q - sk] + ue[q - sk]));
      lw[q] = c.aw / (1. + alfa * (un[q - 1] + ut[q - 1]));
      ls[q] = c.as / (1. + alfa * (ue[q - sj] + ut[q - sj]));
      const double p1 = alfa * (lb[q] * un[q - sk] + lw[q] * un[q - 1]);
      const double p2 = alfa * (lb[q] * ue[q - sk] + ls[q] * ue[q - sj]);
      const double p3 = alfa * (lw[q] * ut[q - 1] + ls[q] * ut[q - sj]);
      lpr[q] = 1. / (ap + p1 + p2 + p3 - lb[q] * ut[q - sk] - lw[q] * ue[q - 1] - ls[q] * un[q - sj] + small);
      un[q] = (c.an - p1) * lpr[q];
      ue[q] = (c.ae - p2) * lpr[q];
      ut[q] = (c.at - p3) * lpr[q];
    });
    __syncthreads();
  }
}

// One SIP sweep of every block (sipsol.for:144-179): residual, forward and
// backward substitution, fi += correction; the block's sum |res| into
// partials[4 * block] (the other three entries zero).
__global__ void __launch_bounds__(512) k_sip_sweep(const BlkLev* __restrict__ bls, SipLU lu, double* __restrict__ fi_all,
                                                   const double* __restrict__ su_all, double* __restrict__ partials) {
  pdl_trigger();
  pdl_wait();
  __shared__ double red[16];
  const BlkLev B = bls[blockIdx.x];
  const double *lb = lu.lb + B.off, *lw = lu.lw + B.off, *ls = lu.ls + B.off, *lpr = lu.lpr + B.off;
  const double *un = lu.un + B.off, *ue = lu.ue + B.off, *ut = lu.ut + B.off;
  double* res = lu.res + B.off;
  double* fi = fi_all + B.off;
  const double* su = su_all + B.off;
  const long long sj = B.sx, sk = B.sxy;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  double acc = 0.0;
  const long long ncell = (long long)nx * ny * nz;
  for (long long c0 = threadIdx.x; c0 < ncell; c0 += blockDim.x) {  // residual, :146-157
    const int x = (int)(c0 % nx) + 1, y = (int)((c0 / nx) % ny) + 1, z = (int)(c0 / ((long long)nx * ny)) + 1;
    const long long q = (long long)z * sk + (long long)y * sj + x;
    const Coef<double> c = cell_coef<double, false>(B, x, y, z, q, nullptr, nullptr, nullptr);
    const double r = (su[q] - coef_ap(c) * fi[q] - c.an * fi[q + sj] - c.as * fi[q - sj] - c.ae * fi[q + 1] -
                      c.aw * fi[q - 1] - c.ab * fi[q - sk] - c.at * fi[q + sk]);
    res[q] = r;
    acc += fabs(r);
  }
  __syncthreads();
  const int dmax = (nx - 1) + (ny - 1) + (nz - 1);
  for (int d = 0; d <= dmax; ++d) {  // forward substitution, :159-167
    sip_plane(B, d, [&](int, int, int, long long q) {
      res[q] = (res[q] - lb[q] * res[q - sk] - lw[q] * res[q - 1] - ls[q] * res[q - sj]) * lpr[q];
    });
    __syncthreads();
  }
  for (int d = dmax; d >= 0; --d) {  // backward substitution and correction, :169-178
    sip_plane(B, d, [&](int, int, int, long long q) {
      res[q] = res[q] - un[q] * res[q + sj] - ue[q] * res[q + 1] - ut[q] * res[q + sk];
      fi[q] = fi[q] + res[q];
    });
    __syncthreads();
  }
  // block sum of |res| in a fixed order (warp shuffles, then warps in order)
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partials[4 * blockIdx.x] = s;
    partials[4 * blockIdx.x + 1] = 0.0;
    partials[4 * blockIdx.x + 2] = 0.0;
    partials[4 * blockIdx.x + 3] = 0.0;
  }
}

__global__ void __launch_bounds__(256) k_gather1(const uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                                 int64_t n, double* __restrict__ a) {
  pdl_trigger();
  pdl_wait();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    a[dst[e]] = a[src[e]];
}

}  // namespace

cudaError_t launch_sip_factor(const BlkLev* bl, int nb, SipArrays a, cudaStream_t st) {
  if (nb <= 0) return cudaSuccess;
  SipLU lu{a.lb, a.lw, a.ls, a.lpr, a.un, a.ue, a.ut, a.res};
  pdl_launch(k_sip_factor, nb, 512, 0, st, bl, lu);
  return cudaGetLastError();
}

cudaError_t launch_sip_sweep(const BlkLev* bl, int nb, SipArrays a, double* fi, const double* su, double* partials,
                             cudaStream_t st) {
  if (nb <= 0) return cudaSuccess;
  SipLU lu{a.lb, a.lw, a.ls, a.lpr, a.un, a.ue, a.ut, a.res};
  pdl_launch(k_sip_sweep, nb, 512, 0, st, bl, lu, fi, su, partials);
  return cudaGetLastError();
}

cudaError_t launch_gather1(const uint32_t* dst, const uint32_t* src, int64_t n, double* a, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  pdl_launch(k_gather1, grid_for(n, 256), 256, 0, st, dst, src, n, a);
  return cudaGetLastError();
}


// The failure path of the bounded waits, made to run out: one warp waits
// (mbar_wait, the sweeps' own routine and limit) on an mbarrier that expects
// one arrival and receives none, so the wait gives up after g_wait_clocks,
// sets *err and the kernel returns.  No copy is issued.
__global__ void k_wait_probe(int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar)) : "memory");
  __syncthreads();
  bool bad = false;
  mbar_wait(smem_u32(&bar), 0u, err, bad);
  __syncthreads();
}

cudaError_t launch_wait_probe(int* err, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(err);
  return cudaGetLastError();
}

cudaError_t set_wait_clocks(long long clocks) {
  const long long c = clocks > 0 ? clocks : (1LL << 26);
  return cudaMemcpyToSymbol(g_wait_clocks, &c, sizeof(c));
}

cudaError_t launch_face_coef_sum(const BlkLev* fine, const BlkLev* coarse, CellTab ct, const double* ffx,
                                 const double* ffy, const double* ffz, double* cfx, double* cfy, double* cfz,
                                 cudaStream_t st) {
  if (ct.ncta <= 0) return cudaSuccess;
  pdl_launch(k_face_coef_sum, ct.ncta, 256, 0, st, fine, coarse, ct.cta_start, ct.nb, ffx, ffy, ffz, cfx, cfy, cfz);
  return cudaGetLastError();
}

cudaError_t launch_calvel(bool lsm, const BlkLev* bl, RowTab rt, const double* h3, const double* p,
                          const double* dens, const double* us, const double* vs, const double* ws, double* u,
                          double* v, double* w, double dtal, cudaStream_t st) {
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = defect_grid(rt.nrows);
  if (lsm) pdl_launch(k_calvel<true>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, h3, p, dens, us, vs, ws, u, v, w, dtal);
  else pdl_launch(k_calvel<false>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, h3, p, dens, us, vs, ws, u, v, w, dtal);
  return cudaGetLastError();
}

cudaError_t launch_gather3(const uint32_t* dst, const uint32_t* src, int64_t n, double* a0, double* a1, double* a2,
                           cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  pdl_launch(k_gather3, grid_for(n, 256), 256, 0, st, dst, src, n, a0, a1, a2);
  return cudaGetLastError();
}

template <typename TR>
cudaError_t launch_calmas(bool lsm, const BlkLev* bl, RowTab rt, const double* h3, const double* u, const double* v,
                          const double* w, double dt, double* bout, TR* rhs_out, double* partials, int* nparts,
                          cudaStream_t st) {
  *nparts = 0;
  if (rt.nrows <= 0) return cudaSuccess;
  const int g = defect_grid(rt.nrows);
  if (lsm) pdl_launch(k_calmas<true, TR>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, h3, u, v, w, dt, bout, rhs_out, partials);
  else pdl_launch(k_calmas<false, TR>, g, 256, 0, st, bl, rt.start, rt.nb, rt.nrows, h3, u, v, w, dt, bout, rhs_out, partials);
  *nparts = g;
  return cudaGetLastError();
}
template cudaError_t launch_calmas<double>(bool, const BlkLev*, RowTab, const double*, const double*, const double*,
                                           const double*, double, double*, double*, double*, int*, cudaStream_t);
template cudaError_t launch_calmas<float>(bool, const BlkLev*, RowTab, const double*, const double*, const double*,
                                          const double*, double, double*, float*, double*, int*, cudaStream_t);

template <typename TE>
cudaError_t launch_padd(const BlkLev* bl, RowTab rt, double* p, const TE* e, cudaStream_t st) {
  if (rt.nrows <= 0) return cudaSuccess;
  pdl_launch(k_padd<TE>, defect_grid(rt.nrows), 256, 0, st, bl, rt.start, rt.nb, rt.nrows, p, e);
  return cudaGetLastError();
}
template cudaError_t launch_padd<double>(const BlkLev*, RowTab, double*, const double*, cudaStream_t);
template cudaError_t launch_padd<float>(const BlkLev*, RowTab, double*, const float*, cudaStream_t);


cudaError_t launch_dens_restrict(const BlkLev* fine, const BlkLev* coarse, CellTab ct, const double* df, double* dc,
                                 cudaStream_t st) {
  if (ct.ncta <= 0) return cudaSuccess;
  pdl_launch(k_dens_restrict, ct.ncta, 256, 0, st, fine, coarse, ct.cta_start, ct.nb, df, dc);
  return cudaGetLastError();
}

cudaError_t launch_face_coef(const BlkLev* bl, CellTab ct, const double* dens, const double* h3, double* fx,
                             double* fy, double* fz, cudaStream_t st) {
  if (ct.ncta <= 0) return cudaSuccess;
  pdl_launch(k_face_coef, ct.ncta, 256, 0, st, bl, ct.cta_start, ct.nb, dens, h3, fx, fy, fz);
  return cudaGetLastError();
}

// explicit instantiations
template cudaError_t launch_rbgs<double>(int, bool, bool, const BlkLev*, const Tile*, int, int, const CUtensorMap*,
                                         const CUtensorMap*, int*, const double*, double*, const double*, const double*, const double*,
                                         const double*, const long long*, float, cudaStream_t);
template cudaError_t launch_rbgs<float>(int, bool, bool, const BlkLev*, const Tile*, int, int, const CUtensorMap*,
                                        const CUtensorMap*, int*, const float*, float*, const float*, const float*, const float*,
                                        const float*, const long long*, float, cudaStream_t);
template cudaError_t launch_fill<double>(const uint32_t*, const uint32_t*, int64_t, double*, const double*,
                                         const double*, bool, cudaStream_t);
template cudaError_t launch_fill<float>(const uint32_t*, const uint32_t*, int64_t, float*, const float*, const float*,
                                        bool, cudaStream_t);
template cudaError_t launch_restrict<double>(bool, bool, const BlkLev*, const BlkLev*, RowTab, const double*,
                                             const double*, double*, const double*, const double*, const double*,
                                             cudaStream_t);
template cudaError_t launch_restrict<float>(bool, bool, const BlkLev*, const BlkLev*, RowTab, const float*,
                                            const float*, float*, const float*, const float*, const float*,
                                            cudaStream_t);
template cudaError_t launch_prolong<double>(bool, const BlkLev*, const BlkLev*, RowTab, const double*, const double*,
                                            double*, cudaStream_t);
template cudaError_t launch_prolong<float>(bool, const BlkLev*, const BlkLev*, RowTab, const float*, const float*,
                                           float*, cudaStream_t);
template cudaError_t launch_defect<double, double>(bool, const BlkLev*, RowTab, const double*, const double*, double*,
                                                   const double*, double*, double, double, const double*,
                                                   const double*, const double*, double*, cudaStream_t);
template cudaError_t launch_defect<float, float>(bool, const BlkLev*, RowTab, const double*, const float*, double*,
                                                 const double*, float*, double, double, const double*, const double*,
                                                 const double*, double*, cudaStream_t);

// ---------------------------------------------------------------------------
// Local mesh refinement (LMR).
//
// Expression fill: the level's exchange sequence, resolved on the host into
// nodes (exchangepp.for LMR branches: 8-cell averages :164-174, injection 2x
// :176-189, the finer receiver's extrapolation :2115-2123, corner and edge
// averages and trilinear values :447-458) evaluated here in the reference's
// operation order.
template <typename T>
__device__ __forceinline__ T xref(uint32_t r, const T* __restrict__ cur, const T* __restrict__ old, bool zero_old,
                                  const T* __restrict__ sc) {
  const uint32_t i = r & 0x3fffffffu;
  switch (r >> 30) {
    case 0: return cur[i];
    case 1: return sc[i];
    case 2: return zero_old ? T(0) : old[i];
    default: return T(0);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_expr_nodes(const uint32_t* __restrict__ nodes, long long begin, long long end,
                                                    const T* __restrict__ cur, const T* __restrict__ old,
                                                    bool zero_old, T* __restrict__ sc) {
  const long long k = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= end) return;
  const uint32_t* w = nodes + 9 * k;
  auto a = [&](int q) { return xref<T>(w[1 + q], cur, old, zero_old, sc); };
  T v;
  switch (w[0]) {
    case 1: {  // 0.125 * (sum of eight), left to right
      T s = a(0);
#pragma unroll
      for (int q = 1; q < 8; ++q) s = s + a(q);
      v = s * T(0.125);
      break;
    }
    case 2: v = T(2) * a(0); break;
    case 3: v = ((a(0) + T(3) * a(1)) - a(2)) * T(0.25); break;  // (r + 3 f1 - f2) / 4
    case 4: {  // (27, 9, 9, 3, 9, 3, 3, 1) / 64, left to right
      T s = T(27) * a(0);
      s = s + T(9) * a(1);
      s = s + T(9) * a(2);
      s = s + T(3) * a(3);
      s = s + T(9) * a(4);
      s = s + T(3) * a(5);
      s = s + T(3) * a(6);
      s = s + a(7);
      v = s * T(1.0 / 64);
      break;
    }
    default: v = a(0); break;
  }
  sc[k] = v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_expr_write(const uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                                    long long n, T* out, const T* cur, const T* __restrict__ sc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  out[dst[e]] = xref<T>(src[e], cur, cur, true, sc);  // writes never read pre-fill values
}

template <typename T>
cudaError_t launch_expr_fill(const uint32_t* nodes, const int64_t* depth_start, int ndepth, const uint32_t* dst,
                             const uint32_t* src, int64_t nw, T* out, const T* cur, const T* old, bool zero_old,
                             T* scratch, cudaStream_t st) {
  for (int d = 0; d < ndepth; ++d) {
    const long long b = depth_start[d], e = depth_start[d + 1];
    if (e <= b) continue;
    k_expr_nodes<T><<<(unsigned)((e - b + 255) / 256), 256, 0, st>>>(nodes, b, e, cur, old, zero_old, scratch);
  }
  if (nw > 0) k_expr_write<T><<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(dst, src, nw, out, cur, scratch);
  return cudaGetLastError();
}
template cudaError_t launch_expr_fill<double>(const uint32_t*, const int64_t*, int, const uint32_t*, const uint32_t*,
                                              int64_t, double*, const double*, const double*, bool, double*,
                                              cudaStream_t);
template cudaError_t launch_expr_fill<float>(const uint32_t*, const int64_t*, int, const uint32_t*, const uint32_t*,
                                             int64_t, float*, const float*, const float*, bool, float*,
                                             cudaStream_t);

// Blocks past their last level: restriction and correction between levels of
// the same size.  Grid (cells / 256, listed blocks); a thread per cell.
template <typename T, bool ZERO>
__global__ void __launch_bounds__(256) k_restrict_same(const BlkLev* __restrict__ fine,
                                                       const BlkLev* __restrict__ coarse, const int* __restrict__ blist,
                                                       const T* __restrict__ phi, const T* __restrict__ rhs,
                                                       T* __restrict__ rhs_c) {
  const int b = blist[blockIdx.y];
  const BlkLev F = fine[b];
  const BlkLev Cc = coarse[b];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= F.nx * F.ny * F.nz) return;
  const int x = 1 + q % F.nx, y = 1 + (q / F.nx) % F.ny, z = 1 + q / (F.nx * F.ny);
  const long long i = F.off + (long long)z * F.sxy + (long long)y * F.sx + x;
  T r = rhs[i];
  if (!ZERO) {
    const Coef<T> c = cell_coef<T, false>(F, x, y, z, i, nullptr, nullptr, nullptr);
    const T ap = coef_ap(c);
    // resf = su - (aw pW + ae pE + as pS + an pN + ab pB + at pT + ap pP), mgsolver.for:706-713
    r = r - (c.aw * phi[i - 1] + c.ae * phi[i + 1] + c.as * phi[i - F.sx] + c.an * phi[i + F.sx] +
             c.ab * phi[i - F.sxy] + c.at * phi[i + F.sxy] + ap * phi[i]);
  }
  rhs_c[Cc.off + (long long)z * Cc.sxy + (long long)y * Cc.sx + x] = r;
}

template <typename T>
cudaError_t launch_restrict_same(bool zero_phi, const BlkLev* fine, const BlkLev* coarse, const int* blist, int nbl,
                                 int max_cells, const T* phi, const T* rhs, T* rhs_c, cudaStream_t st) {
  if (nbl <= 0 || max_cells <= 0) return cudaSuccess;
  dim3 g((unsigned)((max_cells + 255) / 256), (unsigned)nbl);
  if (zero_phi) k_restrict_same<T, true><<<g, 256, 0, st>>>(fine, coarse, blist, phi, rhs, rhs_c);
  else k_restrict_same<T, false><<<g, 256, 0, st>>>(fine, coarse, blist, phi, rhs, rhs_c);
  return cudaGetLastError();
}
template cudaError_t launch_restrict_same<double>(bool, const BlkLev*, const BlkLev*, const int*, int, int,
                                                  const double*, const double*, double*, cudaStream_t);
template cudaError_t launch_restrict_same<float>(bool, const BlkLev*, const BlkLev*, const int*, int, int,
                                                 const float*, const float*, float*, cudaStream_t);

template <typename T, bool ZERO_OLD>
__global__ void __launch_bounds__(256) k_prolong_same(const BlkLev* __restrict__ fine,
                                                      const BlkLev* __restrict__ coarse, const int* __restrict__ blist,
                                                      const T* __restrict__ phi_c, const T* __restrict__ old,
                                                      T* __restrict__ out) {
  const int b = blist[blockIdx.y];
  const BlkLev F = fine[b];
  const BlkLev Cc = coarse[b];
  const int mx = F.nx + 2, my = F.ny + 2;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= mx * my * (F.nz + 2)) return;
  const int x = q % mx, y = (q / mx) % my, z = q / (mx * my);
  // mgbound after the correction: a wall ghost takes its neighbour's corrected value
  const int ph = F.phys;
  int sx = x, sy = y, sz = z;
  if (x == 0 && (ph & 1)) sx = 1;
  if (x == F.nx + 1 && (ph & 2)) sx = F.nx;
  if (y == 0 && (ph & 4)) sy = 1;
  if (y == F.ny + 1 && (ph & 8)) sy = F.ny;
  if (z == 0 && (ph & 16)) sz = 1;
  if (z == F.nz + 1 && (ph & 32)) sz = F.nz;
  const T o = ZERO_OLD ? T(0) : old[F.off + (long long)sz * F.sxy + (long long)sy * F.sx + sx];
  out[F.off + (long long)z * F.sxy + (long long)y * F.sx + x] =
      o + phi_c[Cc.off + (long long)sz * Cc.sxy + (long long)sy * Cc.sx + sx];
}

template <typename T>
cudaError_t launch_prolong_same(bool zero_old, const BlkLev* fine, const BlkLev* coarse, const int* blist, int nbl,
                                int max_cells, const T* phi_c, const T* old, T* out, cudaStream_t st) {
  if (nbl <= 0 || max_cells <= 0) return cudaSuccess;
  dim3 g((unsigned)((max_cells + 255) / 256), (unsigned)nbl);
  if (zero_old) k_prolong_same<T, true><<<g, 256, 0, st>>>(fine, coarse, blist, phi_c, old, out);
  else k_prolong_same<T, false><<<g, 256, 0, st>>>(fine, coarse, blist, phi_c, old, out);
  return cudaGetLastError();
}
template cudaError_t launch_prolong_same<double>(bool, const BlkLev*, const BlkLev*, const int*, int, int,
                                                 const double*, const double*, double*, cudaStream_t);
template cudaError_t launch_prolong_same<float>(bool, const BlkLev*, const BlkLev*, const int*, int, int,
                                                const float*, const float*, float*, cudaStream_t);

}  // namespace h3d
