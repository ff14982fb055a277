// Internal declarations shared by the host runtime (h3d_mg.cu), the halo
// table builder (h3d_halo.cpp) and the kernels (h3d_kernels.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/h3d_mg.h"

namespace h3d {

constexpr int kMaxLevels = 16;
constexpr uint32_t kOldFlag = 0x80000000u;  // halo entry reads the pre-fill value
constexpr uint32_t kIdxMask = 0x7fffffffu;
constexpr int kRowAlign = 4;     // row pitch multiple (elements): 16 B for FP32, 32 B for FP64
constexpr int kBlockAlign = 64;  // block base multiple (elements)
// Padded device layout: x = 0 of every row sits kXOff elements after a 16-byte
// boundary, so the first interior cell x = 1 starts on one (vector loads and
// stores of 4 FP32 / 2 FP64 cells).  TMA boxes start at that boundary (x = -3).
constexpr int kXOff = 3;

// Per-(block, level) geometry as the kernels see it.  Cell (x,y,z), 0-based
// with the ghost layer at 0 and n+1, lives at off + z*sxy + y*sx + x.
struct BlkLev {
  int nx, ny, nz;       // interior cells
  int sx;               // row pitch (>= nx+2; padded on the device)
  long long sxy;        // plane pitch sx*(ny+2)
  long long off;        // element offset of cell (0,0,0) in the level array
  int phys;             // bit f set: face f (W,E,S,N,B,T) is a physical non-periodic wall
  int pad;
  double ax, ay, az;    // constant coefficients 1/dxx, 1/dyy, 1/dzz (mgsolver.for:54-60,186-191)
  double dv;            // cell volume at level 1 (dx*dy*dz), for the rmax measure
};

// Tile of the smoother / cell kernels: block, first interior x, y, z of the tile.
struct Tile {
  int b, x0, y0, z0;
};

// Level geometry in the canonical packed numbering.
struct LevelGeom {
  int g = 0;
  std::vector<BlkLev> bl;
  // local mesh refinement: block past its last level here (g > ngrid, its
  // restriction into this level is a copy), and block whose next coarser level
  // has this level's size (g >= ngrid, its correction from it is an add)
  std::vector<char> clamped, same_next;
  int64_t n_elems = 0;      // total cells incl. ghosts
  int64_t n_interior = 0;   // total interior cells
};

// Builds the level geometry from block descriptors (level dims with the
// reference's clamp, mgsolver.for:392-400).  pad: the device layout (aligned
// row pitch and block bases); otherwise the canonical dense numbering.
LevelGeom make_level_geom(const std::vector<h3d_block_desc>& blocks, int g, bool pad);

// Halo gather tables (see h3d_halo_table in h3d_mg.h).
enum HaloKind { kHaloSweep = 0, kHaloExchange = 1, kHaloBound = 2, kHaloFaces = 3 };
int build_halo_table(const std::vector<h3d_block_desc>& blocks, int g, int kind, bool pad,
                     std::vector<uint32_t>& dst, std::vector<uint32_t>& src,
                     std::string* err);

// Local mesh refinement (LMR): rdv(ib, g) of every block at level g
// (localparameters.for:44-59), from the descriptors' rdiv and ngrid.
std::vector<int> level_rdv(const std::vector<h3d_block_desc>& blocks, int g);
// True when some face, edge or corner neighbours differ in rdv at level g:
// the level's fill then has arithmetic (averages, injections, extrapolation,
// trilinear values) and is built as an expression table.
bool level_is_lmr(const std::vector<h3d_block_desc>& blocks, int g);

// Expression form of a level's ghost fill.  A reference (32 bits) is, by its
// two top bits: 0 the current value of a cell, 2 (kOldFlag) the pre-fill value
// of a cell, 1 (kRefNode) the value of node i, 3 (kRefZero) zero.  Nodes are
// 9 words (op, up to 8 operand references) and sorted by depth: a node reads
// cells and nodes of lower depth only.  Every ghost write reads a current
// cell, a node or zero, never a pre-fill value, so the writes may run in
// place.
constexpr uint32_t kRefNode = 0x40000000u;
constexpr uint32_t kRefZero = 0xC0000000u;
constexpr uint32_t kRefMask = 0x3fffffffu;
enum ExprOp : uint32_t {
  kXCopy = 0,      // a
  kXAvg8 = 1,      // (a0 + a1 + ... + a7) * 0.125, summed left to right
  kXInj2 = 2,      // 2 * a
  kXExtrap = 3,    // ((a0 + 3 a1) - a2) / 4
  kXInterp64 = 4,  // (27 a0 + 9 a1 + 9 a2 + 3 a3 + 9 a4 + 3 a5 + 3 a6 + 1 a7) / 64, left to right
};
struct ExprTable {
  std::vector<uint32_t> nodes;        // 9 words a node
  std::vector<int64_t> depth_start;   // node ranges of depth 0, 1, ...: [depth_start[d], depth_start[d+1])
  std::vector<uint32_t> dst, src;     // ghost writes: cell dst <- reference src
};
int build_expr_table(const std::vector<h3d_block_desc>& blocks, int g, int kind, bool pad, ExprTable& X,
                     std::string* err);

// Error text of a call that has no handle (read with h3d_mg_last_error(NULL)).
void set_call_error(const std::string& msg);

}  // namespace h3d
