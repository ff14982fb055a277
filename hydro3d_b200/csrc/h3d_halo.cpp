// Halo gather tables: the ghost-cell semantics of the reference's level
// exchange, resolved on index arrays so the GPU can fill every ghost cell of
// a level in one order-free gather.
//
// The reference fills MG ghosts with a fixed sequence of plane, edge and
// corner copies: mgbound (mgsolver.for:912-997), then exchangepp
// (exchangepp.for:44-2826: per direction a pack pass over all blocks then an
// unpack pass; corners and edges with the z direction), then mgbound again
// (:2830) and the periodic wrap exchbc_mgpp (:2832, :2837-3454).  Running
// that sequence on cell *identities* instead of values gives, for every
// ghost cell, the cell whose value it ends up holding.  When that source is
// an interior cell the GPU gathers the current value; when it is a ghost (a
// value the sequence never replaced) the GPU reads the pre-fill value, which
// the out-of-place smoother keeps in the previous buffer.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <initializer_list>

#include "h3d_internal.h"

namespace h3d {

LevelGeom make_level_geom(const std::vector<h3d_block_desc>& blocks, int g, bool pad) {
  LevelGeom L;
  L.g = g;
  long long off = 0;
  for (const auto& d : blocks) {
    int gl = g > d.ngrid ? d.ngrid : g;  // mgsolver.for:392-396
    BlkLev b{};
    b.nx = d.n[0] >> (gl - 1);
    b.ny = d.n[1] >> (gl - 1);
    b.nz = d.n[2] >> (gl - 1);
    // padded layout: row pitch a multiple of 16 bytes (TMA global strides),
    // x = 1 of every row on a 16-byte boundary (block base = 256-byte boundary
    // + kXOff); the canonical layout is dense.
    b.sx = pad ? ((b.nx + 2 + kXOff + kRowAlign - 1) / kRowAlign) * kRowAlign : b.nx + 2;
    b.sxy = (long long)b.sx * (b.ny + 2);
    if (pad) off = (off + kBlockAlign - 1) / kBlockAlign * kBlockAlign + kXOff;
    b.off = off;
    b.phys = 0;
    for (int f = 0; f < 6; ++f)
      if (d.nb_face[f] < 0 && d.bc[f] != 5) b.phys |= 1 << f;
    double s = (double)(1 << (gl - 1));
    double ndx = d.h[0] * s, ndy = d.h[1] * s, ndz = d.h[2] * s;
    double dxx = ndx * ndx, dyy = ndy * ndy, dzz = ndz * ndz;
    b.ax = 1.0 / dxx;
    b.ay = 1.0 / dyy;
    b.az = 1.0 / dzz;
    b.dv = d.h[0] * d.h[1] * d.h[2];
    off += b.sxy * (b.nz + 2);
    L.n_interior += (int64_t)b.nx * b.ny * b.nz;
    L.bl.push_back(b);
    L.clamped.push_back(g > d.ngrid);
    L.same_next.push_back(g >= d.ngrid);
  }
  L.n_elems = off;
  return L;
}

namespace {

struct Emu {
  const LevelGeom& L;
  const std::vector<h3d_block_desc>& D;
  std::vector<uint32_t> id;
  Emu(const LevelGeom& l, const std::vector<h3d_block_desc>& d) : L(l), D(d), id((size_t)l.n_elems) {
    for (size_t q = 0; q < id.size(); ++q) id[q] = (uint32_t)q;
  }
  size_t at(int b, int x, int y, int z) const {
    const BlkLev& B = L.bl[b];
    return (size_t)(B.off + (long long)z * B.sxy + (long long)y * B.sx + x);
  }
  int n(int b, int a) const { return a == 0 ? L.bl[b].nx : (a == 1 ? L.bl[b].ny : L.bl[b].nz); }
  // Cell of block b whose coordinate on axis a is c and whose other two
  // coordinates are (u, v) in axis order.
  size_t plane_cell(int b, int a, int c, int u, int v) const {
    if (a == 0) return at(b, c, u, v);
    if (a == 1) return at(b, u, c, v);
    return at(b, u, v, c);
  }
  void read_plane(int b, int a, int c, std::vector<uint32_t>& buf) const {
    int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
    int n1 = n(b, o1) + 2, n2 = n(b, o2) + 2;
    buf.resize((size_t)n1 * n2);
    for (int v = 0; v < n2; ++v)
      for (int u = 0; u < n1; ++u) buf[(size_t)v * n1 + u] = id[plane_cell(b, a, c, u, v)];
  }
  bool write_plane(int b, int a, int c, const std::vector<uint32_t>& buf) {
    int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
    int n1 = n(b, o1) + 2, n2 = n(b, o2) + 2;
    if (buf.size() != (size_t)n1 * n2) return false;  // face neighbours must match
    for (int v = 0; v < n2; ++v)
      for (int u = 0; u < n1; ++u) id[plane_cell(b, a, c, u, v)] = buf[(size_t)v * n1 + u];
    return true;
  }
  void copy_plane(int b, int a, int cdst, int csrc) {
    int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
    int n1 = n(b, o1) + 2, n2 = n(b, o2) + 2;
    for (int v = 0; v < n2; ++v)
      for (int u = 0; u < n1; ++u) id[plane_cell(b, a, cdst, u, v)] = id[plane_cell(b, a, csrc, u, v)];
  }

  // mgbound: zero-gradient ghosts on physical faces, order W,E,S,N,B,T.
  void mgbound() {
    for (size_t b = 0; b < L.bl.size(); ++b) {
      int phys = L.bl[b].phys;
      for (int a = 0; a < 3; ++a) {
        if (phys & (1 << (2 * a))) copy_plane((int)b, a, 0, 1);
        if (phys & (1 << (2 * a + 1))) copy_plane((int)b, a, n((int)b, a) + 1, n((int)b, a));
      }
    }
  }

  // Coordinate codes for corner/edge cells: 0 -> ghost 0, 1 -> first interior,
  // 2 -> last interior (n), 3 -> ghost n+1, 4 -> running index.
  int coord(int code, int nn, int running) const {
    switch (code) {
      case 0: return 0;
      case 1: return 1;
      case 2: return nn;
      case 3: return nn + 1;
      default: return running;
    }
  }

  bool exchangepp(std::string* err) {
    // Corner cells (exchangepp.for:441-640, 1400-1600 pack; 2515-2718 unpack),
    // as (sender cell, receiver cell) for prev #1..4 then next #1..4.
    static const int csrc[8][3] = {{1, 1, 1}, {1, 2, 1}, {2, 2, 1}, {2, 1, 1},
                                   {2, 2, 2}, {2, 1, 2}, {1, 1, 2}, {1, 2, 2}};
    static const int cdst[8][3] = {{0, 0, 0}, {0, 3, 0}, {3, 3, 0}, {3, 0, 0},
                                   {3, 3, 3}, {3, 0, 3}, {0, 0, 3}, {0, 3, 3}};
    // Edges (exchangepp.for:646-1100, 1604-2056 pack; 2568-2826 unpack).
    static const int eaxis[6] = {1, 0, 1, 0, 2, 2};
    static const int esrc[12][3] = {{1, 4, 1}, {4, 2, 1}, {2, 4, 1}, {4, 1, 1}, {1, 1, 4}, {1, 2, 4},
                                    {2, 4, 2}, {4, 1, 2}, {1, 4, 2}, {4, 2, 2}, {2, 2, 4}, {2, 1, 4}};
    static const int edst[12][3] = {{0, 4, 0}, {4, 3, 0}, {3, 4, 0}, {4, 0, 0}, {0, 0, 4}, {0, 3, 4},
                                    {3, 4, 3}, {4, 0, 3}, {0, 4, 3}, {4, 3, 3}, {3, 3, 4}, {3, 0, 4}};
    const int nb = (int)L.bl.size();
    std::vector<std::vector<uint32_t>> rm(nb), rp(nb);
    std::vector<uint32_t> rc(nb * 8, 0);
    std::vector<char> rc_set(nb * 8, 0);
    std::vector<std::vector<uint32_t>> re((size_t)nb * 12);
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < nb; ++b) {  // pack
        int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        if (prev >= 0) read_plane(b, a, 1, rp[prev]);
        if (a == 2) {
          for (int c = 0; c < 4; ++c) {
            int t = D[b].nb_corner[c];
            if (t < 0) continue;
            // receiver slot: sender's prev corner c lands in the receiver's next slot c
            rc[t * 8 + 4 + c] = id[at(b, coord(csrc[c][0], L.bl[b].nx, 0), coord(csrc[c][1], L.bl[b].ny, 0),
                                      coord(csrc[c][2], L.bl[b].nz, 0))];
            rc_set[t * 8 + 4 + c] = 1;
          }
          for (int e = 0; e < 6; ++e) {
            int t = D[b].nb_edge[e];
            if (t < 0) continue;
            int len = n(b, eaxis[e]);
            auto& buf = re[(size_t)t * 12 + 6 + e];
            buf.assign(len + 2, 0);
            for (int q = 1; q <= len; ++q)
              buf[q] = id[at(b, coord(esrc[e][0], L.bl[b].nx, q), coord(esrc[e][1], L.bl[b].ny, q),
                             coord(esrc[e][2], L.bl[b].nz, q))];
          }
        }
        if (next >= 0) read_plane(b, a, n(b, a), rm[next]);
        if (a == 2) {
          for (int c = 0; c < 4; ++c) {
            int t = D[b].nb_corner[4 + c];
            if (t < 0) continue;
            rc[t * 8 + c] = id[at(b, coord(csrc[4 + c][0], L.bl[b].nx, 0), coord(csrc[4 + c][1], L.bl[b].ny, 0),
                                  coord(csrc[4 + c][2], L.bl[b].nz, 0))];
            rc_set[t * 8 + c] = 1;
          }
          for (int e = 0; e < 6; ++e) {
            int t = D[b].nb_edge[6 + e];
            if (t < 0) continue;
            int len = n(b, eaxis[e]);
            auto& buf = re[(size_t)t * 12 + e];
            buf.assign(len + 2, 0);
            for (int q = 1; q <= len; ++q)
              buf[q] = id[at(b, coord(esrc[6 + e][0], L.bl[b].nx, q), coord(esrc[6 + e][1], L.bl[b].ny, q),
                             coord(esrc[6 + e][2], L.bl[b].nz, q))];
          }
        }
      }
      for (int b = 0; b < nb; ++b) {  // unpack
        int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        if (prev >= 0 && !write_plane(b, a, 0, rm[b])) {
          if (err) *err = "face neighbours with different extents";
          return false;
        }
        if (next >= 0 && !write_plane(b, a, n(b, a) + 1, rp[b])) {
          if (err) *err = "face neighbours with different extents";
          return false;
        }
        if (a == 2) {
          const BlkLev& B = L.bl[b];
          for (int c = 0; c < 4; ++c)  // prev corners (filled by the neighbour's next pack)
            if (D[b].nb_corner[c] >= 0 && rc_set[b * 8 + c])
              id[at(b, coord(cdst[c][0], B.nx, 0), coord(cdst[c][1], B.ny, 0), coord(cdst[c][2], B.nz, 0))] =
                  rc[b * 8 + c];
          for (int e = 0; e < 6; ++e)
            if (D[b].nb_edge[e] >= 0) {
              auto& buf = re[(size_t)b * 12 + e];
              int len = n(b, eaxis[e]);
              if ((int)buf.size() != len + 2) {
                if (err) *err = "edge neighbours with different extents";
                return false;
              }
              for (int q = 1; q <= len; ++q)
                id[at(b, coord(edst[e][0], B.nx, q), coord(edst[e][1], B.ny, q), coord(edst[e][2], B.nz, q))] =
                    buf[q];
            }
          for (int c = 0; c < 4; ++c)  // next corners
            if (D[b].nb_corner[4 + c] >= 0 && rc_set[b * 8 + 4 + c])
              id[at(b, coord(cdst[4 + c][0], B.nx, 0), coord(cdst[4 + c][1], B.ny, 0),
                    coord(cdst[4 + c][2], B.nz, 0))] = rc[b * 8 + 4 + c];
          for (int e = 0; e < 6; ++e)
            if (D[b].nb_edge[6 + e] >= 0) {
              auto& buf = re[(size_t)b * 12 + 6 + e];
              int len = n(b, eaxis[e]);
              if ((int)buf.size() != len + 2) {
                if (err) *err = "edge neighbours with different extents";
                return false;
              }
              for (int q = 1; q <= len; ++q)
                id[at(b, coord(edst[6 + e][0], B.nx, q), coord(edst[6 + e][1], B.ny, q),
                      coord(edst[6 + e][2], B.nz, q))] = buf[q];
            }
        }
      }
    }
    mgbound();
    bool periodic = false;
    for (int b = 0; b < nb; ++b)
      for (int f = 0; f < 6; ++f)
        if (D[b].bc[f] == 5) periodic = true;
    if (periodic) return exchbc(err);
    return true;
  }

  bool exchbc(std::string* err) {
    const int nb = (int)L.bl.size();
    std::vector<std::vector<uint32_t>> rm(nb), rp(nb);
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < nb; ++b) {
        if (!(D[b].bc[2 * a] == 5 || D[b].bc[2 * a + 1] == 5)) continue;
        int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        int na = n(b, a);
        if (prev < 0) {
          if (next < 0) copy_plane(b, a, 0, na);
          else if (D[b].nb_periodic[2 * a] >= 0) read_plane(b, a, 1, rp[D[b].nb_periodic[2 * a]]);
        }
        if (next < 0) {
          if (prev < 0) copy_plane(b, a, na + 1, 1);
          else if (D[b].nb_periodic[2 * a + 1] >= 0) read_plane(b, a, na, rm[D[b].nb_periodic[2 * a + 1]]);
        }
      }
      for (int b = 0; b < nb; ++b) {
        if (!(D[b].bc[2 * a] == 5 || D[b].bc[2 * a + 1] == 5)) continue;
        int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        if (prev < 0 && next >= 0 && D[b].nb_periodic[2 * a] >= 0 && !write_plane(b, a, 0, rm[b])) {
          if (err) *err = "periodic partners with different extents";
          return false;
        }
        if (next < 0 && prev >= 0 && D[b].nb_periodic[2 * a + 1] >= 0 &&
            !write_plane(b, a, n(b, a) + 1, rp[b])) {
          if (err) *err = "periodic partners with different extents";
          return false;
        }
      }
    }
    return true;
  }

  // ---- local mesh refinement: the exchange on references with arithmetic ----
  // Node storage (9 words a node, see ExprTable); node refs carry kRefNode.
  std::vector<uint32_t> nodes;
  std::vector<int> rdv;  // per block at this level

  uint32_t mk(uint32_t op, std::initializer_list<uint32_t> a) {
    const uint32_t k = (uint32_t)(nodes.size() / 9);
    nodes.push_back(op);
    int q = 0;
    for (uint32_t v : a) { nodes.push_back(v); ++q; }
    for (; q < 8; ++q) nodes.push_back(kRefZero);
    return k | kRefNode;
  }
  // 1-based, ghost-inclusive (i, j, k) of the reference (ghost at 1 and n)
  size_t c1(int b, int i, int j, int k) const { return at(b, i - 1, j - 1, k - 1); }
  int n1(int b, int a) const { return n(b, a) + 2; }
  // face plane of direction a as (c, u, w): (j,k) for a = 0, (i,k) for 1, (j,i) for 2
  size_t fc(int b, int a, int c, int u, int w) const {
    if (a == 0) return c1(b, c, u, w);
    if (a == 1) return c1(b, u, c, w);
    return c1(b, w, u, c);
  }
  int ns1(int b, int a) const { return a == 1 ? n1(b, 0) : n1(b, 1); }
  int ns2(int b, int a) const { return a == 2 ? n1(b, 0) : n1(b, 2); }
  int cmp(int b, int t) const { return rdv[b] == rdv[t] ? 0 : (rdv[b] > rdv[t] ? 1 : -1); }

  // exchangepp.for:149-430 / 1107-1393 (pack) and 2101-2505 (unpack), same
  // rank: equal resolution copies the full plane; a finer sender averages its
  // 2x2x2 cells onto the coarse plane interior; a coarser sender injects twice
  // its cell into four fine entries, which the finer receiver extrapolates
  // with its own first two planes over the full plane.
  void face_pack(int b, int a, bool prev, int c, std::vector<uint32_t>& rb) {
    const int s1 = ns1(b, a), s2 = ns2(b, a), na = n1(b, a);
    if (c == 0) {
      const int cc = prev ? 2 : na - 1;
      for (int w = 1; w <= s2; ++w)
        for (int u = 1; u <= s1; ++u) rb[(size_t)(w - 1) * s1 + u] = id[fc(b, a, cc, u, w)];
    } else if (c > 0) {
      const int sc1 = (s1 - 2) / 2 + 2, sc2 = (s2 - 2) / 2 + 2, c0 = prev ? 2 : na - 2;
      for (int w = 2; w <= sc2 - 1; ++w)
        for (int u = 2; u <= sc1 - 1; ++u) {
          const int u0 = 2 * u - 2, w0 = 2 * w - 2;
          rb[(size_t)(w - 1) * sc1 + u] =
              mk(kXAvg8, {id[fc(b, a, c0, u0, w0)], id[fc(b, a, c0, u0 + 1, w0)], id[fc(b, a, c0, u0, w0 + 1)],
                          id[fc(b, a, c0, u0 + 1, w0 + 1)], id[fc(b, a, c0 + 1, u0, w0)],
                          id[fc(b, a, c0 + 1, u0 + 1, w0)], id[fc(b, a, c0 + 1, u0, w0 + 1)],
                          id[fc(b, a, c0 + 1, u0 + 1, w0 + 1)]});
        }
    } else {
      const int sr1 = 2 * (s1 - 2) + 2, cc = prev ? 2 : na - 1;
      for (int w = 2; w <= s2 - 1; ++w)
        for (int u = 2; u <= s1 - 1; ++u) {
          const uint32_t v = mk(kXInj2, {id[fc(b, a, cc, u, w)]});
          rb[(size_t)(2 * w - 3) * sr1 + 2 * u - 2] = v;
          rb[(size_t)(2 * w - 3) * sr1 + 2 * u - 1] = v;
          rb[(size_t)(2 * w - 2) * sr1 + 2 * u - 2] = v;
          rb[(size_t)(2 * w - 2) * sr1 + 2 * u - 1] = v;
        }
    }
  }
  void face_unpack(int b, int a, bool prev, int c, const std::vector<uint32_t>& rb) {
    const int s1 = ns1(b, a), s2 = ns2(b, a), na = n1(b, a);
    const int cg = prev ? 1 : na, f1 = prev ? 2 : na - 1, f2 = prev ? 3 : na - 2;
    if (c == 0) {
      for (int w = 1; w <= s2; ++w)
        for (int u = 1; u <= s1; ++u) id[fc(b, a, cg, u, w)] = rb[(size_t)(w - 1) * s1 + u];
    } else if (c > 0) {
      for (int w = 1; w <= s2; ++w)
        for (int u = 1; u <= s1; ++u)
          id[fc(b, a, cg, u, w)] =
              mk(kXExtrap, {rb[(size_t)(w - 1) * s1 + u], id[fc(b, a, f1, u, w)], id[fc(b, a, f2, u, w)]});
    } else {
      for (int w = 2; w <= s2 - 1; ++w)
        for (int u = 2; u <= s1 - 1; ++u) id[fc(b, a, cg, u, w)] = rb[(size_t)(w - 1) * s1 + u];
    }
  }
  // Corner and edge cells of a sender: per axis the code 1 (first interior),
  // 2 (last interior) or 4 (running), as in exchangepp() above.
  // The 2x2x2 average of a finer sender, j then i then k as the fastest bit
  // (exchangepp.for:447-451); the trilinear value of a coarser sender from
  // its cell and the neighbours toward the receiver, same bit order
  // (:452-458).
  uint32_t avg8(int b, int i0, int j0, int k0) {
    return mk(kXAvg8, {id[c1(b, i0, j0, k0)], id[c1(b, i0, j0 + 1, k0)], id[c1(b, i0 + 1, j0, k0)],
                       id[c1(b, i0 + 1, j0 + 1, k0)], id[c1(b, i0, j0, k0 + 1)], id[c1(b, i0, j0 + 1, k0 + 1)],
                       id[c1(b, i0 + 1, j0, k0 + 1)], id[c1(b, i0 + 1, j0 + 1, k0 + 1)]});
  }
  uint32_t interp64(int b, int i0, int j0, int k0, int si, int sj, int sk) {
    return mk(kXInterp64, {id[c1(b, i0, j0, k0)], id[c1(b, i0, j0 + sj, k0)], id[c1(b, i0 + si, j0, k0)],
                           id[c1(b, i0 + si, j0 + sj, k0)], id[c1(b, i0, j0, k0 + sk)],
                           id[c1(b, i0, j0 + sj, k0 + sk)], id[c1(b, i0 + si, j0, k0 + sk)],
                           id[c1(b, i0 + si, j0 + sj, k0 + sk)]});
  }
  // sender cell (1-based) of code cd on axis a, running index r (1-based)
  int spos(int b, int a, int cd, int r) const { return cd == 4 ? r : (cd == 1 ? 2 : n1(b, a) - 1); }
  int sbase(int b, int a, int cd, int r) const { return cd == 4 ? r : (cd == 1 ? 2 : n1(b, a) - 2); }
  int sout(int cd) const { return cd == 1 ? -1 : 1; }
  uint32_t corner_val(int b, const int* cd, int c) {
    if (c == 0) return id[c1(b, spos(b, 0, cd[0], 0), spos(b, 1, cd[1], 0), spos(b, 2, cd[2], 0))];
    if (c > 0) return avg8(b, sbase(b, 0, cd[0], 0), sbase(b, 1, cd[1], 0), sbase(b, 2, cd[2], 0));
    return interp64(b, spos(b, 0, cd[0], 0), spos(b, 1, cd[1], 0), spos(b, 2, cd[2], 0), sout(cd[0]), sout(cd[1]),
                    sout(cd[2]));
  }
  // exchangepp.for:646-1100, 1604-2056: buf is indexed 1-based like re1p(nn)
  void edge_val(int b, const int* cd, int ax, int c, std::vector<uint32_t>& buf) {
    const int len = n1(b, ax);
    if (c == 0) {
      for (int r = 2; r <= len - 1; ++r)
        buf[r] = id[c1(b, spos(b, 0, cd[0], r), spos(b, 1, cd[1], r), spos(b, 2, cd[2], r))];
    } else if (c > 0) {
      const int lenc = (len - 2) / 2 + 2;
      for (int r = 2; r <= lenc - 1; ++r)
        buf[r] = avg8(b, sbase(b, 0, cd[0], 2 * r - 2), sbase(b, 1, cd[1], 2 * r - 2), sbase(b, 2, cd[2], 2 * r - 2));
    } else {
      for (int r = 2; r <= len - 1; ++r)
        for (int hh = 0; hh < 2; ++hh) {
          int sg[3];
          for (int a = 0; a < 3; ++a) sg[a] = cd[a] == 4 ? (hh ? 1 : -1) : sout(cd[a]);
          buf[2 * r - 2 + hh] = interp64(b, spos(b, 0, cd[0], r), spos(b, 1, cd[1], r), spos(b, 2, cd[2], r), sg[0],
                                         sg[1], sg[2]);
        }
    }
  }

  bool exchangepp_lmr(std::string* err) {
    static const int csrc[8][3] = {{1, 1, 1}, {1, 2, 1}, {2, 2, 1}, {2, 1, 1},
                                   {2, 2, 2}, {2, 1, 2}, {1, 1, 2}, {1, 2, 2}};
    static const int cdst[8][3] = {{0, 0, 0}, {0, 3, 0}, {3, 3, 0}, {3, 0, 0},
                                   {3, 3, 3}, {3, 0, 3}, {0, 0, 3}, {0, 3, 3}};
    static const int eaxis[6] = {1, 0, 1, 0, 2, 2};
    static const int esrc[12][3] = {{1, 4, 1}, {4, 2, 1}, {2, 4, 1}, {4, 1, 1}, {1, 1, 4}, {1, 2, 4},
                                    {2, 4, 2}, {4, 1, 2}, {1, 4, 2}, {4, 2, 2}, {2, 2, 4}, {2, 1, 4}};
    static const int edst[12][3] = {{0, 4, 0}, {4, 3, 0}, {3, 4, 0}, {4, 0, 0}, {0, 0, 4}, {0, 3, 4},
                                    {3, 4, 3}, {4, 0, 3}, {0, 4, 3}, {4, 3, 3}, {3, 3, 4}, {3, 0, 4}};
    const int nb = (int)L.bl.size();
    size_t ngg = 0;
    for (int b = 0; b < nb; ++b) {
      const size_t x = n1(b, 0), y = n1(b, 1), z = n1(b, 2);
      ngg = std::max(ngg, std::max(x * y, std::max(x * z, y * z)));
    }
    // the reference's receive buffers: entries no sender of this call writes
    // hold an earlier exchange's values; here they read as zero
    std::vector<std::vector<uint32_t>> rbm(nb, std::vector<uint32_t>(ngg + 1, kRefZero)),
        rbp(nb, std::vector<uint32_t>(ngg + 1, kRefZero));
    std::vector<uint32_t> rc(nb * 8, kRefZero);
    std::vector<char> rc_set(nb * 8, 0);
    std::vector<std::vector<uint32_t>> re((size_t)nb * 12);
    for (int b = 0; b < nb; ++b)
      for (int e = 0; e < 12; ++e) re[(size_t)b * 12 + e].assign(n1(b, eaxis[e % 6]) + 1, kRefZero);
    for (int b = 0; b < nb; ++b) {  // neighbours differ by at most a factor of 2
      for (int f = 0; f < 6; ++f) {
        const int t = D[b].nb_face[f];
        if (t >= 0 && (rdv[b] > 2 * rdv[t] || rdv[t] > 2 * rdv[b])) {
          if (err) *err = "face neighbours differ by more than a factor of 2 in refinement";
          return false;
        }
      }
      for (int e = 0; e < 12; ++e) {
        const int t = D[b].nb_edge[e];
        if (t >= 0 && (rdv[b] > 2 * rdv[t] || rdv[t] > 2 * rdv[b])) {
          if (err) *err = "edge neighbours differ by more than a factor of 2 in refinement";
          return false;
        }
      }
      for (int c = 0; c < 8; ++c) {
        const int t = D[b].nb_corner[c];
        if (t >= 0 && (rdv[b] > 2 * rdv[t] || rdv[t] > 2 * rdv[b])) {
          if (err) *err = "corner neighbours differ by more than a factor of 2 in refinement";
          return false;
        }
      }
    }
    auto code1 = [&](int b, int a, int cd, int r) {  // receiver cell, codes 0, 3 (ghosts), 4 (running)
      return cd == 0 ? 1 : (cd == 3 ? n1(b, a) : r);
    };
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < nb; ++b) {  // pack
        const int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        if (prev >= 0) face_pack(b, a, true, cmp(b, prev), rbp[prev]);
        if (a == 2) {
          for (int c = 0; c < 4; ++c) {
            const int t = D[b].nb_corner[c];
            if (t >= 0) {
              rc[t * 8 + 4 + c] = corner_val(b, csrc[c], cmp(b, t));
              rc_set[t * 8 + 4 + c] = 1;
            }
          }
          for (int e = 0; e < 6; ++e) {
            const int t = D[b].nb_edge[e];
            if (t >= 0) edge_val(b, esrc[e], eaxis[e], cmp(b, t), re[(size_t)t * 12 + 6 + e]);
          }
        }
        if (next >= 0) face_pack(b, a, false, cmp(b, next), rbm[next]);
        if (a == 2) {
          for (int c = 0; c < 4; ++c) {
            const int t = D[b].nb_corner[4 + c];
            if (t >= 0) {
              rc[t * 8 + c] = corner_val(b, csrc[4 + c], cmp(b, t));
              rc_set[t * 8 + c] = 1;
            }
          }
          for (int e = 0; e < 6; ++e) {
            const int t = D[b].nb_edge[6 + e];
            if (t >= 0) edge_val(b, esrc[6 + e], eaxis[e], cmp(b, t), re[(size_t)t * 12 + e]);
          }
        }
      }
      for (int b = 0; b < nb; ++b) {  // unpack
        const int prev = D[b].nb_face[2 * a], next = D[b].nb_face[2 * a + 1];
        if (prev >= 0) face_unpack(b, a, true, cmp(b, prev), rbm[b]);
        if (next >= 0) face_unpack(b, a, false, cmp(b, next), rbp[b]);
        if (a == 2) {  // corners and edges: plain copies at every resolution (:2511-2826)
          for (int c = 0; c < 4; ++c)
            if (D[b].nb_corner[c] >= 0 && rc_set[b * 8 + c])
              id[c1(b, code1(b, 0, cdst[c][0], 0), code1(b, 1, cdst[c][1], 0), code1(b, 2, cdst[c][2], 0))] =
                  rc[b * 8 + c];
          for (int e = 0; e < 6; ++e)
            if (D[b].nb_edge[e] >= 0) {
              const auto& buf = re[(size_t)b * 12 + e];
              for (int r = 2; r <= n1(b, eaxis[e]) - 1; ++r)
                id[c1(b, code1(b, 0, edst[e][0], r), code1(b, 1, edst[e][1], r), code1(b, 2, edst[e][2], r))] =
                    buf[r];
            }
          for (int c = 0; c < 4; ++c)
            if (D[b].nb_corner[4 + c] >= 0 && rc_set[b * 8 + 4 + c])
              id[c1(b, code1(b, 0, cdst[4 + c][0], 0), code1(b, 1, cdst[4 + c][1], 0),
                    code1(b, 2, cdst[4 + c][2], 0))] = rc[b * 8 + 4 + c];
          for (int e = 0; e < 6; ++e)
            if (D[b].nb_edge[6 + e] >= 0) {
              const auto& buf = re[(size_t)b * 12 + 6 + e];
              for (int r = 2; r <= n1(b, eaxis[e]) - 1; ++r)
                id[c1(b, code1(b, 0, edst[6 + e][0], r), code1(b, 1, edst[6 + e][1], r),
                      code1(b, 2, edst[6 + e][2], r))] = buf[r];
            }
        }
      }
    }
    mgbound();
    bool periodic = false;
    for (int b = 0; b < nb; ++b)
      for (int f = 0; f < 6; ++f)
        if (D[b].bc[f] == 5) periodic = true;
    if (periodic) return exchbc(err);
    return true;
  }

  bool is_interior(uint32_t q) const {
    // find block by offset (blocks are sorted by offset)
    size_t lo = 0, hi = L.bl.size();
    while (hi - lo > 1) {
      size_t mid = (lo + hi) / 2;
      if ((uint64_t)L.bl[mid].off <= q) lo = mid;
      else hi = mid;
    }
    const BlkLev& B = L.bl[lo];
    long long r = (long long)q - B.off;
    int z = (int)(r / B.sxy);
    long long t = r - (long long)z * B.sxy;
    int y = (int)(t / B.sx);
    int x = (int)(t - (long long)y * B.sx);
    return x >= 1 && x <= B.nx && y >= 1 && y <= B.ny && z >= 1 && z <= B.nz;
  }
};

}  // namespace

int build_halo_table(const std::vector<h3d_block_desc>& blocks, int g, int kind, bool pad,
                     std::vector<uint32_t>& dst, std::vector<uint32_t>& src, std::string* err) {
  LevelGeom L = make_level_geom(blocks, g, pad);
  if (L.n_elems >= (int64_t)kOldFlag) {
    if (err) *err = "level too large for 31-bit halo indices";
    return H3D_ERR_BAD_CONFIG;
  }
  Emu E(L, blocks);
  bool ok = true;
  switch (kind) {
    case kHaloSweep:
    case kHaloFaces:
      E.mgbound();
      ok = E.exchangepp(err);
      break;
    case kHaloExchange:
      ok = E.exchangepp(err);
      break;
    case kHaloBound:
      E.mgbound();
      break;
    default:
      if (err) *err = "unknown halo kind";
      return H3D_ERR_ARG;
  }
  if (!ok) return H3D_ERR_BAD_CONFIG;
  dst.clear();
  src.clear();
  for (size_t b = 0; b < L.bl.size(); ++b) {
    const BlkLev& B = L.bl[b];
    for (int z = 0; z <= B.nz + 1; ++z)
      for (int y = 0; y <= B.ny + 1; ++y)
        for (int x = 0; x <= B.nx + 1; ++x) {
          int outside = (x == 0 || x == B.nx + 1) + (y == 0 || y == B.ny + 1) + (z == 0 || z == B.nz + 1);
          if (outside == 0) {
            // interior cells are never written by the fill; x jumps across the row
            if (x == 0) continue;
            x = B.nx;  // skip to the east ghost
            continue;
          }
          if (kind == kHaloFaces && outside != 1) continue;
          size_t q = E.at((int)b, x, y, z);
          uint32_t s = E.id[q];
          bool inter = E.is_interior(s);
          if (kind == kHaloFaces) {
            if (!inter) {
              if (err) *err = "face ghost without an interior source";
              return H3D_ERR_INTERNAL;
            }
            if (s == (uint32_t)q) continue;
          }
          dst.push_back((uint32_t)q);
          src.push_back(inter ? s : (s | kOldFlag));
        }
  }
  return H3D_OK;
}

std::vector<int> level_rdv(const std::vector<h3d_block_desc>& blocks, int g) {
  // ngrid_input = ngrid - log2(rdiv), the same for every block (checked at create)
  std::vector<int> r(blocks.size(), 1);
  for (size_t b = 0; b < blocks.size(); ++b) {
    const h3d_block_desc& d = blocks[b];
    int lg = 0;
    while ((1 << lg) < d.rdiv) ++lg;
    const int ngi = d.ngrid - lg;
    if (g > d.ngrid) r[b] = 1;
    else if (g <= ngi) r[b] = d.rdiv > 0 ? d.rdiv : 1;
    else r[b] = (d.rdiv > 0 ? d.rdiv : 1) >> (g - ngi);
  }
  return r;
}

bool level_is_lmr(const std::vector<h3d_block_desc>& blocks, int g) {
  const std::vector<int> r = level_rdv(blocks, g);
  for (size_t b = 0; b < blocks.size(); ++b) {
    const h3d_block_desc& d = blocks[b];
    for (int f = 0; f < 6; ++f)
      if (d.nb_face[f] >= 0 && r[d.nb_face[f]] != r[b]) return true;
    for (int e = 0; e < 12; ++e)
      if (d.nb_edge[e] >= 0 && r[d.nb_edge[e]] != r[b]) return true;
    for (int c = 0; c < 8; ++c)
      if (d.nb_corner[c] >= 0 && r[d.nb_corner[c]] != r[b]) return true;
  }
  return false;
}

int build_expr_table(const std::vector<h3d_block_desc>& blocks, int g, int kind, bool pad, ExprTable& X,
                     std::string* err) {
  LevelGeom L = make_level_geom(blocks, g, pad);
  if (L.n_elems > (int64_t)kRefMask) {
    if (err) *err = "level too large for 30-bit expression references";
    return H3D_ERR_BAD_CONFIG;
  }
  Emu E(L, blocks);
  E.rdv = level_rdv(blocks, g);
  bool ok = true;
  switch (kind) {
    case kHaloSweep:
      E.mgbound();
      ok = E.exchangepp_lmr(err);
      break;
    case kHaloExchange:
      ok = E.exchangepp_lmr(err);
      break;
    case kHaloBound:
      E.mgbound();
      break;
    default:
      if (err) *err = "expression tables are built for the sweep, exchange and bound fills";
      return H3D_ERR_ARG;
  }
  if (!ok) return H3D_ERR_BAD_CONFIG;
  // cell references: interior cells read the current value, ghosts the pre-fill one
  auto leaf = [&](uint32_t r) -> uint32_t {
    if ((r & ~kRefMask) != 0) return r;  // node or zero
    return E.is_interior(r) ? r : (r | kOldFlag);
  };
  const size_t nn = E.nodes.size() / 9;
  // ghost writes first (a write from a pre-fill value becomes a copy node)
  std::vector<uint32_t> wd, ws;
  for (size_t b = 0; b < L.bl.size(); ++b) {
    const BlkLev& B = L.bl[b];
    for (int z = 0; z <= B.nz + 1; ++z)
      for (int y = 0; y <= B.ny + 1; ++y)
        for (int x = 0; x <= B.nx + 1; ++x) {
          const int outside = (x == 0 || x == B.nx + 1) + (y == 0 || y == B.ny + 1) + (z == 0 || z == B.nz + 1);
          if (outside == 0) {
            if (x == 0) continue;
            x = B.nx;
            continue;
          }
          const size_t q = E.at((int)b, x, y, z);
          uint32_t r = leaf(E.id[q]);
          if ((r & ~kRefMask) == kOldFlag) r = E.mk(kXCopy, {r & kRefMask});
          wd.push_back((uint32_t)q);
          ws.push_back(r);
        }
  }
  // operands of the nodes made above and of the copy nodes
  const size_t nall = E.nodes.size() / 9;
  std::vector<int> depth(nall, 0);
  int maxd = 0;
  for (size_t k = 0; k < nall; ++k) {
    int dk = 0;
    for (int q = 1; q <= 8; ++q) {
      uint32_t& r = E.nodes[9 * k + q];
      if (k >= nn && q == 1 && E.nodes[9 * k] == kXCopy) {
        r = r | kOldFlag;  // copy node of a pre-fill value (leaf() already applied)
        continue;
      }
      r = leaf(r);
      if ((r & ~kRefMask) == kRefNode) dk = std::max(dk, depth[r & kRefMask] + 1);
    }
    depth[k] = dk;
    maxd = std::max(maxd, dk);
  }
  // depth-sorted order, stable
  std::vector<uint32_t> order(nall), newidx(nall);
  {
    std::vector<int64_t> cnt(maxd + 2, 0);
    for (size_t k = 0; k < nall; ++k) ++cnt[depth[k] + 1];
    for (int d = 1; d <= maxd + 1; ++d) cnt[d] += cnt[d - 1];
    X.depth_start.assign(cnt.begin(), cnt.end());
    for (size_t k = 0; k < nall; ++k) {
      const int64_t p = cnt[depth[k]]++;
      order[p] = (uint32_t)k;
      newidx[k] = (uint32_t)p;
    }
  }
  auto remap = [&](uint32_t r) { return (r & ~kRefMask) == kRefNode ? (newidx[r & kRefMask] | kRefNode) : r; };
  X.nodes.assign(9 * nall, 0);
  for (size_t p = 0; p < nall; ++p) {
    const size_t k = order[p];
    X.nodes[9 * p] = E.nodes[9 * k];
    for (int q = 1; q <= 8; ++q) X.nodes[9 * p + q] = remap(E.nodes[9 * k + q]);
  }
  X.dst = wd;
  X.src.resize(ws.size());
  for (size_t e = 0; e < ws.size(); ++e) X.src[e] = remap(ws[e]);
  return H3D_OK;
}

}  // namespace h3d

extern "C" int h3d_halo_expr(int32_t nblocks, const h3d_block_desc* blocks, int32_t g, int32_t kind,
                             uint32_t* nodes, int64_t node_cap, int64_t* nnodes, uint32_t* dst, uint32_t* src,
                             int64_t cap, int64_t* n) {
  if (!blocks || nblocks <= 0 || g < 1 || !n || !nnodes) return H3D_ERR_ARG;
  std::vector<h3d_block_desc> D(blocks, blocks + nblocks);
  for (auto& d : D)
    if (g > d.ngrid + 8 || d.ngrid < 1) return H3D_ERR_ARG;
  h3d::ExprTable X;
  int rc = h3d::build_expr_table(D, g, kind, false, X, nullptr);
  if (rc != H3D_OK) return rc;
  *n = (int64_t)X.dst.size();
  *nnodes = (int64_t)X.nodes.size() / 9;
  if (dst && src) {
    if (cap < *n) return H3D_ERR_ARG;
    std::memcpy(dst, X.dst.data(), X.dst.size() * sizeof(uint32_t));
    std::memcpy(src, X.src.data(), X.src.size() * sizeof(uint32_t));
  }
  if (nodes) {
    if (node_cap < *nnodes) return H3D_ERR_ARG;
    std::memcpy(nodes, X.nodes.data(), X.nodes.size() * sizeof(uint32_t));
  }
  return H3D_OK;
}

extern "C" int h3d_halo_table(int32_t nblocks, const h3d_block_desc* blocks, int32_t g, int32_t kind,
                              uint32_t* dst, uint32_t* src, int64_t cap, int64_t* n) {
  if (!blocks || nblocks <= 0 || g < 1 || !n) return H3D_ERR_ARG;
  std::vector<h3d_block_desc> D(blocks, blocks + nblocks);
  for (auto& d : D)
    if (g > d.ngrid || d.ngrid < 1) return H3D_ERR_ARG;
  std::vector<uint32_t> vd, vs;
  int rc = h3d::build_halo_table(D, g, kind, false, vd, vs, nullptr);
  if (rc != H3D_OK) return rc;
  *n = (int64_t)vd.size();
  if (dst && src) {
    if (cap < (int64_t)vd.size()) return H3D_ERR_ARG;
    std::memcpy(dst, vd.data(), vd.size() * sizeof(uint32_t));
    std::memcpy(src, vs.data(), vs.size() * sizeof(uint32_t));
  }
  return H3D_OK;
}
