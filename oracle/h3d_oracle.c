/*
 * h3d_oracle.c -- CPU oracle (test infrastructure only; see h3d_oracle.h).
 *
 * A restatement in C of the reference multigrid path of Hydro3D v7.0:
 *   coeff, mgkcyc, mgrelax, mgrestr, mgcorr, mgbound   (src_v70/mgsolver.for)
 *   exchangepp, exchbc_mgpp (same-rank branches, incl. the local mesh
 *   refinement ones between blocks of refinement ratio 1:2)
 *                                                      (src_v70/exchangepp.for)
 *   rdv(ib,g) and per-block level counts of LMR       (src_v70/localparameters.for:24-59)
 *   newsolv_mg outer loop                              (src_v70/newsolv_mg.for)
 *   read_infodom neighbour discovery                   (src_v70/alloc_dom.for)
 * All arithmetic is IEEE FP64 evaluated left to right in the reference's
 * operand order; build with -ffp-contract=off so no FMA is formed.
 *
 * Index conventions follow the reference: i,j,k are 1-based and include the
 * one ghost layer (interior 2..n-1); `cof` is 1-based and the level-g phi
 * slab is j-fastest: (k-1)*ni*nj + (i-1)*nj + j + faz(g) - ni*nj*nk
 * (mgsolver.for:412); coefficient slot s of cell (i,j,k) lives at
 * faz(g) + (k-2)(ni-2)(nj-2) + (i-2)(nj-2) + (j-1) + s*incr (mgsolver.for:413-420).
 */
#include "h3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXLEV 16

typedef struct {
  or_block_desc d;
  int ngrid;
  int64_t faz[MAXLEV + 1];      /* faz(1..ngrd) as in mgsolver.for:23-41 */
  int64_t nwork;
  double* cof;                  /* 1-based, cof[1..nwork] */
  double* dens;                 /* interior density (nz,ny,nx) x-fastest */
  double* dens_mg;              /* 1-based dens_mg(1..tot) */
  int64_t ijkp_lsm[MAXLEV + 1]; /* initial.for:203-213 */
  /* same-rank receive buffers of exchangepp (1-based) */
  double* recvb_m1;
  double* recvb_p1;
  double rc_m[5], rc_p[5];      /* rc1m..rc4m, rc1p..rc4p */
  double* re_m[7];              /* re1m..re6m */
  double* re_p[7];              /* re1p..re6p */
} or_dom;

struct or_mg {
  int nbp, ngrd_gl, mg_itrsch, irestr, iproln, lsm, periodic;
  int ngg;                      /* longest line / largest plane */
  int err;
  int lmr;                      /* some blocks have rdiv > 1 */
  int* rdv;                     /* rdv(ib, g) at rdv[ib * (MAXLEV + 1) + g] */
  or_dom* dom;
};
#define RDV(m, ib, g) ((m)->rdv[(ib) * (MAXLEV + 1) + (g)])

static int g_threads = 1;
void or_set_threads(int n) { g_threads = n > 0 ? n : 1; }

static int ipow2(int e) { return 1 << e; }

/* Level dims incl. ghosts with the reference's level clamp
 * (mgsolver.for:392-400). */
static void lev_dims(const or_dom* d, int g, int* ni, int* nj, int* nk) {
  int gl = g > d->ngrid ? d->ngrid : g;
  *ni = d->d.n[0] / ipow2(gl - 1) + 2;
  *nj = d->d.n[1] / ipow2(gl - 1) + 2;
  *nk = d->d.n[2] / ipow2(gl - 1) + 2;
}

/* phi index (1-based) of cell (i,j,k) of level g. */
#define PHI(i, j, k) ((int64_t)((k)-1) * nij + (int64_t)((i)-1) * nj + (j) + nijk)

or_mg* or_create(int nblocks, const or_block_desc* blocks, int ngrd_gl,
                 int mg_itrsch, int irestr, int iproln, int lsm) {
  or_mg* m = (or_mg*)calloc(1, sizeof(or_mg));
  m->nbp = nblocks;
  m->ngrd_gl = ngrd_gl;
  m->mg_itrsch = mg_itrsch;
  m->irestr = irestr;
  m->iproln = iproln;
  m->lsm = lsm;
  m->dom = (or_dom*)calloc((size_t)nblocks, sizeof(or_dom));
  m->rdv = (int*)calloc((size_t)nblocks * (MAXLEV + 1), sizeof(int));
  if (ngrd_gl < 1 || ngrd_gl > MAXLEV) m->err = 1;
  /* localparameters.for:28-59: ngrd_gl = ngrid_input + log2(max rdiv); a block
   * of ratio rdiv has ngrid_input + log2(rdiv) levels; rdv(ib, g) is rdiv up to
   * level ngrid_input, halves on each further level of the block, and is 1
   * beyond the block's last level. */
  int maxlog = 0;
  for (int ib = 0; ib < nblocks; ++ib) {
    int r = blocks[ib].rdiv, lg = 0;
    while ((1 << lg) < r) ++lg;
    if (r < 1 || (1 << lg) != r) m->err = 1;
    if (lg > maxlog) maxlog = lg;
    if (r > 1) m->lmr = 1;
  }
  int ngrid_input = ngrd_gl - maxlog;
  if (ngrid_input < 1) m->err = 1;
  int nmax = 0;
  for (int ib = 0; ib < nblocks; ++ib) {
    or_dom* d = &m->dom[ib];
    d->d = blocks[ib];
    d->ngrid = blocks[ib].ngrid;
    int lg = 0;
    while ((1 << lg) < blocks[ib].rdiv) ++lg;
    if (d->ngrid != ngrid_input + lg) m->err = 1;
    if (m->err) continue;
    for (int g = 1; g <= ngrd_gl; ++g) {
      int v;
      if (g > d->ngrid) v = 1;
      else if (g <= ngrid_input) v = blocks[ib].rdiv;
      else v = RDV(m, ib, g - 1) / 2;
      RDV(m, ib, g) = v;
    }
    for (int a = 0; a < 6; ++a)
      if (d->d.bc[a] == 5) m->periodic = 1; /* alloc_dom.for:1224-1231 */
    /* divisibility check, localparameters.for:204-209 */
    int pow2 = ipow2(d->ngrid - 1);
    for (int a = 0; a < 3; ++a)
      if (d->d.n[a] <= 0 || d->d.n[a] % pow2 != 0) m->err = 1;
    if (m->err) continue;
    /* nwork, localparameters.for:226-236 */
    int64_t nwork = 0;
    for (int g = 1; g <= ngrd_gl; ++g) {
      int ni, nj, nk;
      lev_dims(d, g, &ni, &nj, &nk);
      nwork += (int64_t)ni * nj * nk + 8LL * (ni - 2) * (nj - 2) * (nk - 2);
    }
    d->nwork = nwork;
    d->cof = (double*)calloc((size_t)nwork + 1, sizeof(double));
    int ni = d->d.n[0] + 2, nj = d->d.n[1] + 2, nk = d->d.n[2] + 2;
    int pmax = ni * nj;
    if (ni * nk > pmax) pmax = ni * nk;
    if (nj * nk > pmax) pmax = nj * nk;
    if (pmax > nmax) nmax = pmax;
    /* ijkp_lsm, initial.for:203-213 */
    d->ijkp_lsm[0] = 0;
    for (int g = 1; g <= d->ngrid; ++g) {
      int a, b, c;
      lev_dims(d, g, &a, &b, &c);
      d->ijkp_lsm[g] = d->ijkp_lsm[g - 1] + (int64_t)(a - 2) * (b - 2) * (c - 2);
    }
    d->dens_mg = (double*)calloc((size_t)d->ijkp_lsm[d->ngrid] + 1, sizeof(double));
    d->dens = (double*)calloc((size_t)d->d.n[0] * d->d.n[1] * d->d.n[2], sizeof(double));
    for (int64_t q = 0; q < (int64_t)d->d.n[0] * d->d.n[1] * d->d.n[2]; ++q) d->dens[q] = 1.0;
  }
  m->ngg = nmax;
  for (int ib = 0; ib < nblocks && !m->err; ++ib) {
    or_dom* d = &m->dom[ib];
    d->recvb_m1 = (double*)calloc((size_t)nmax + 1, sizeof(double));
    d->recvb_p1 = (double*)calloc((size_t)nmax + 1, sizeof(double));
    int lmax = d->d.n[0] + 2;
    if (d->d.n[1] + 2 > lmax) lmax = d->d.n[1] + 2;
    if (d->d.n[2] + 2 > lmax) lmax = d->d.n[2] + 2;
    for (int e = 1; e <= 6; ++e) {
      d->re_m[e] = (double*)calloc((size_t)lmax + 1, sizeof(double));
      d->re_p[e] = (double*)calloc((size_t)lmax + 1, sizeof(double));
    }
  }
  return m;
}

int or_error(const or_mg* m) { return m->err; }

void or_destroy(or_mg* m) {
  if (!m) return;
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    free(d->cof);
    free(d->dens);
    free(d->dens_mg);
    free(d->recvb_m1);
    free(d->recvb_p1);
    for (int e = 1; e <= 6; ++e) {
      free(d->re_m[e]);
      free(d->re_p[e]);
    }
  }
  free(m->dom);
  free(m->rdv);
  free(m);
}

void or_set_density(or_mg* m, int ib, const double* dens) {
  or_dom* d = &m->dom[ib];
  memcpy(d->dens, dens, sizeof(double) * (size_t)d->d.n[0] * d->d.n[1] * d->d.n[2]);
}

/* dens(i+pl-1, j+pl-1, k+pl-1) for the 1-based ghost-inclusive level-1 index
 * (mgsolver.for:82) == interior cell (i-2, j-2, k-2). */
static double dens_at(const or_dom* d, int i, int j, int k) {
  return d->dens[((int64_t)(k - 2) * d->d.n[1] + (j - 2)) * d->d.n[0] + (i - 2)];
}

/* ------------------------------------------------------------------ coeff */
void or_coeff(or_mg* m) { /* mgsolver.for:2-224 */
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    if (m->lsm)
      for (int64_t q = 0; q <= d->ijkp_lsm[d->ngrid]; ++q) d->dens_mg[q] = 0.0;
    int pi, pj, pk;
    lev_dims(d, 1, &pi, &pj, &pk);
    d->faz[1] = (int64_t)pi * pj * pk; /* :23-28 */
    for (int glevel = 2; glevel <= m->ngrd_gl; ++glevel) { /* :29-41 */
      int ci, cj, ck;
      lev_dims(d, glevel, &ci, &cj, &ck);
      d->faz[glevel] = d->faz[glevel - 1] + (int64_t)ci * cj * ck +
                       8LL * (pi - 2) * (pj - 2) * (pk - 2);
      pi = ci; pj = cj; pk = ck;
    }
    const int* nb = d->d.nb_face;
    const int* bc = d->d.bc;
    for (int glevel = 1; glevel <= m->ngrd_gl; ++glevel) { /* :44 */
      int gl = glevel > d->ngrid ? d->ngrid : glevel;
      int mi, mj, mk;
      lev_dims(d, glevel, &mi, &mj, &mk);
      double ndx = d->d.h[0] * ipow2(gl - 1);
      double ndy = d->d.h[1] * ipow2(gl - 1);
      double ndz = d->d.h[2] * ipow2(gl - 1);
      double dxx = ndx * ndx, dyy = ndy * ndy, dzz = ndz * ndz;
      int64_t cnt = d->faz[glevel] - (int64_t)mi * mj * mk; /* :62-70 */
      for (int64_t q = 1; q <= (int64_t)mi * mj * mk; ++q) d->cof[cnt + q] = 0.0;

      if (m->lsm) { /* :72-112 dens_mg hierarchy */
        for (int k = 2; k <= mk - 1; ++k)
          for (int i = 2; i <= mi - 1; ++i)
            for (int j = 2; j <= mj - 1; ++j) {
              if (glevel == 1) {
                int64_t q = (int64_t)(k - 2) * (mi - 2) * (mj - 2) + (int64_t)(i - 2) * (mj - 2) + (j - 1);
                d->dens_mg[q] = dens_at(d, i, j, k);
              } else {
                int64_t q = d->ijkp_lsm[glevel - 1] + (int64_t)(k - 2) * (mi - 2) * (mj - 2) +
                            (int64_t)(i - 2) * (mj - 2) + (j - 1);
                int pni = d->d.n[0] / ipow2(glevel - 2) + 2;
                int pnj = d->d.n[1] / ipow2(glevel - 2) + 2;
                int64_t ij1 = (int64_t)(2 * k - 4) * (pni - 2) * (pnj - 2) + (int64_t)(2 * i - 4) * (pnj - 2) +
                              (2 * j - 3) + d->ijkp_lsm[glevel - 2];
                int64_t ij2 = ij1 + 1, ij3 = ij1 + (pnj - 2), ij4 = ij1 + (pnj - 2) + 1;
                int64_t pl2 = (int64_t)(pni - 2) * (pnj - 2);
                int64_t ij5 = ij1 + pl2, ij6 = ij1 + pl2 + 1, ij7 = ij1 + pl2 + (pnj - 2),
                        ij8 = ij1 + pl2 + (pnj - 2) + 1;
                double* dm = d->dens_mg;
                d->dens_mg[q] = 0.125 * (dm[ij1] + dm[ij2] + dm[ij3] + dm[ij4] + dm[ij5] + dm[ij6] +
                                         dm[ij7] + dm[ij8]);
              }
            }
      }

      int64_t incr = (int64_t)(mi - 2) * (mj - 2) * (mk - 2); /* :114 */
      for (int k = 2; k <= mk - 1; ++k)
        for (int i = 2; i <= mi - 1; ++i)
          for (int j = 2; j <= mj - 1; ++j) {
            int64_t ijk = d->faz[glevel] + (int64_t)(k - 2) * (mi - 2) * (mj - 2) +
                          (int64_t)(i - 2) * (mj - 2) + (j - 1);
            double* c = d->cof;
            if (m->lsm) { /* :122-184 */
              int64_t q = (glevel == 1 ? 0 : d->ijkp_lsm[glevel - 1]) +
                          (int64_t)(k - 2) * (mi - 2) * (mj - 2) + (int64_t)(i - 2) * (mj - 2) + (j - 1);
              const double* dm = d->dens_mg;
              int64_t sx = (mj - 2), sz = (int64_t)(mi - 2) * (mj - 2);
              double dim = (i == 2) ? dm[q] : 0.5 * (dm[q] + dm[q - sx]);
              double dip = (i == mi - 1) ? dm[q] : 0.5 * (dm[q] + dm[q + sx]);
              double djm = (j == 2) ? dm[q] : 0.5 * (dm[q] + dm[q - 1]);
              double djp = (j == mj - 1) ? dm[q] : 0.5 * (dm[q] + dm[q + 1]);
              double dkm = (k == 2) ? dm[q] : 0.5 * (dm[q] + dm[q - sz]);
              double dkp = (k == mk - 1) ? dm[q] : 0.5 * (dm[q] + dm[q + sz]);
              double dx = d->d.h[0], dy = d->d.h[1], dz = d->d.h[2];
              c[ijk] = dy * dz / dx / dim;
              c[ijk + 1 * incr] = dy * dz / dx / dip;
              c[ijk + 2 * incr] = dx * dz / dy / djm;
              c[ijk + 3 * incr] = dx * dz / dy / djp;
              c[ijk + 4 * incr] = dx * dy / dz / dkm;
              c[ijk + 5 * incr] = dx * dy / dz / dkp;
            } else { /* :186-191 */
              c[ijk] = 1.0 / dxx;
              c[ijk + 1 * incr] = 1.0 / dxx;
              c[ijk + 2 * incr] = 1.0 / dyy;
              c[ijk + 3 * incr] = 1.0 / dyy;
              c[ijk + 4 * incr] = 1.0 / dzz;
              c[ijk + 5 * incr] = 1.0 / dzz;
            }
            /* physical, non-periodic faces, :194-205 */
            if (nb[0] < 0 && bc[0] != 5 && i == 2) c[ijk] = 0.0;
            if (nb[1] < 0 && bc[1] != 5 && i == mi - 1) c[ijk + 1 * incr] = 0.0;
            if (nb[2] < 0 && bc[2] != 5 && j == 2) c[ijk + 2 * incr] = 0.0;
            if (nb[3] < 0 && bc[3] != 5 && j == mj - 1) c[ijk + 3 * incr] = 0.0;
            if (nb[4] < 0 && bc[4] != 5 && k == 2) c[ijk + 4 * incr] = 0.0;
            if (nb[5] < 0 && bc[5] != 5 && k == mk - 1) c[ijk + 5 * incr] = 0.0;
            c[ijk + 6 * incr] = -1.0 * (c[ijk] + c[ijk + 1 * incr] + c[ijk + 2 * incr] +
                                        c[ijk + 3 * incr] + c[ijk + 4 * incr] + c[ijk + 5 * incr]);
            c[ijk + 7 * incr] = 0.0;
          }
    }
  }
}

/* ------------------------------------------------------------- accessors */
void or_put_phi(or_mg* m, int g, int ib, const double* a) {
  or_dom* d = &m->dom[ib];
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
  for (int k = 1; k <= nk; ++k)
    for (int i = 1; i <= ni; ++i)
      for (int j = 1; j <= nj; ++j)
        d->cof[PHI(i, j, k)] = a[((int64_t)(k - 1) * nj + (j - 1)) * ni + (i - 1)];
}

void or_get_phi(const or_mg* m, int g, int ib, double* a) {
  const or_dom* d = &m->dom[ib];
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i)
        a[((int64_t)(k - 1) * nj + (j - 1)) * ni + (i - 1)] = d->cof[PHI(i, j, k)];
}

static int64_t cofidx(const or_dom* d, int g, int ni, int nj, int i, int j, int k) {
  return d->faz[g] + (int64_t)(k - 2) * (ni - 2) * (nj - 2) + (int64_t)(i - 2) * (nj - 2) + (j - 1);
}

void or_get_coef(const or_mg* m, int g, int ib, int s, double* a) {
  const or_dom* d = &m->dom[ib];
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t incr = (int64_t)(ni - 2) * (nj - 2) * (nk - 2);
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        a[((int64_t)(k - 2) * (nj - 2) + (j - 2)) * (ni - 2) + (i - 2)] =
            d->cof[cofidx(d, g, ni, nj, i, j, k) + s * incr];
}

/* Multiplies the seven coefficient slots (aw..ap) of level g by s.  Not a
 * reference routine: it models the product's consistent coarse-level
 * scaling of the L_LSM coefficients (s = 4^-(g-1)), under which the coarse
 * correction of the FV-integrated operator is the consistent one instead of
 * 4^-(g-1) of it (coeff uses the fine dx, dy, dz on every level,
 * mgsolver.for:130-184). */
void or_scale_level_coef(or_mg* m, int g, double s) {
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    int ni, nj, nk;
    lev_dims(d, g, &ni, &nj, &nk);
    int64_t incr = (int64_t)(ni - 2) * (nj - 2) * (nk - 2);
    for (int64_t q = 0; q < 7 * incr; ++q) d->cof[d->faz[g] + 1 + q] *= s;
  }
}

/* Overwrites coefficient slot s of level g (interior, x fastest).  Not a
 * reference routine: lets tests model the product's coarse operators. */
void or_set_coef(or_mg* m, int g, int ib, int s, const double* a) {
  or_dom* d = &m->dom[ib];
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t incr = (int64_t)(ni - 2) * (nj - 2) * (nk - 2);
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        d->cof[cofidx(d, g, ni, nj, i, j, k) + s * incr] =
            a[((int64_t)(k - 2) * (nj - 2) + (j - 2)) * (ni - 2) + (i - 2)];
}

void or_put_rhs(or_mg* m, int g, int ib, const double* a) {
  or_dom* d = &m->dom[ib];
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t incr = (int64_t)(ni - 2) * (nj - 2) * (nk - 2);
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
  for (int k = 2; k <= nk - 1; ++k)
    for (int i = 2; i <= ni - 1; ++i)
      for (int j = 2; j <= nj - 1; ++j)
        d->cof[cofidx(d, g, ni, nj, i, j, k) + 7 * incr] =
            a[((int64_t)(k - 2) * (nj - 2) + (j - 2)) * (ni - 2) + (i - 2)];
}

void or_get_rhs(const or_mg* m, int g, int ib, double* a) {
  or_get_coef(m, g, ib, 7, a);
}

/* ---------------------------------------------------------------- mgbound */
void or_mgbound(or_mg* m, int g) { /* mgsolver.for:912-997 */
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    int ni, nj, nk;
    lev_dims(d, g, &ni, &nj, &nk);
    int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
    double* c = d->cof;
    const int* nb = d->d.nb_face;
    const int* bc = d->d.bc;
    if (nb[0] < 0 && bc[0] != 5)
      for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j) c[PHI(1, j, k)] = c[PHI(1, j, k) + nj];
    if (nb[1] < 0 && bc[1] != 5)
      for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j) c[PHI(ni, j, k)] = c[PHI(ni, j, k) - nj];
    if (nb[2] < 0 && bc[2] != 5)
      for (int k = 1; k <= nk; ++k)
        for (int i = 1; i <= ni; ++i) c[PHI(i, 1, k)] = c[PHI(i, 1, k) + 1];
    if (nb[3] < 0 && bc[3] != 5)
      for (int k = 1; k <= nk; ++k)
        for (int i = 1; i <= ni; ++i) c[PHI(i, nj, k)] = c[PHI(i, nj, k) - 1];
    if (nb[4] < 0 && bc[4] != 5)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) c[PHI(i, j, 1)] = c[PHI(i, j, 1) + nij];
    if (nb[5] < 0 && bc[5] != 5)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) c[PHI(i, j, nk)] = c[PHI(i, j, nk) - nij];
  }
}

/* ------------------------------------------------------------- exchangepp */
/* Corner and edge cells: pack position in the sender and unpack position in
 * the receiver, as 1-based ghost-inclusive (i,j,k) with 0 = "1", -1 = "n-1",
 * -2 = "n", 2 = "2" and 99 = "running index nn" (exchangepp.for:441-1100,
 * 1400-2056 pack; 2511-2826 unpack). */
enum { P2 = 2, PN1 = -1, PN = -2, P1 = 1, RUN = 99 };
static int pos(int code, int n, int nn) {
  switch (code) {
    case P1: return 1;
    case P2: return 2;
    case PN1: return n - 1;
    case PN: return n;
    default: return nn;
  }
}
/* prev corners #1..4: sender cell -> receiver's rcNp -> receiver cell */
static const int corprev_src[4][3] = {{P2, P2, P2}, {P2, PN1, P2}, {PN1, PN1, P2}, {PN1, P2, P2}};
static const int cornext_src[4][3] = {{PN1, PN1, PN1}, {PN1, P2, PN1}, {P2, P2, PN1}, {P2, PN1, PN1}};
/* unpack of rcNm (prev corners of the receiver), exchangepp.for:2515-2566 */
static const int corprev_dst[4][3] = {{P1, P1, P1}, {P1, PN, P1}, {PN, PN, P1}, {PN, P1, P1}};
/* unpack of rcNp (next corners of the receiver), exchangepp.for:2668-2718 */
static const int cornext_dst[4][3] = {{PN, PN, PN}, {PN, P1, PN}, {P1, P1, PN}, {P1, PN, PN}};
/* edges: axis that runs (0 i, 1 j, 2 k) and the fixed positions */
static const int edg_axis[6] = {1, 0, 1, 0, 2, 2};
static const int edgprev_src[6][3] = {{P2, RUN, P2}, {RUN, PN1, P2}, {PN1, RUN, P2},
                                      {RUN, P2, P2}, {P2, P2, RUN}, {P2, PN1, RUN}};
static const int edgnext_src[6][3] = {{PN1, RUN, PN1}, {RUN, P2, PN1}, {P2, RUN, PN1},
                                      {RUN, PN1, PN1}, {PN1, PN1, RUN}, {PN1, P2, RUN}};
static const int edgprev_dst[6][3] = {{P1, RUN, P1}, {RUN, PN, P1}, {PN, RUN, P1},
                                      {RUN, P1, P1}, {P1, P1, RUN}, {P1, PN, RUN}};
static const int edgnext_dst[6][3] = {{PN, RUN, PN}, {RUN, P1, PN}, {P1, RUN, PN},
                                      {RUN, PN, PN}, {PN, PN, RUN}, {PN, P1, RUN}};

static int edge_len(int e, int ni, int nj, int nk) {
  int ax = edg_axis[e];
  return ax == 0 ? ni : (ax == 1 ? nj : nk);
}

/* Level view of one block for the exchange: dims incl. ghosts and the phi
 * slab offsets of mgsolver.for:412. */
typedef struct {
  int n[3];            /* ni, nj, nk */
  int64_t nij, nj, nijk;
  double* fi;
} lview;

static lview lview_of(or_mg* m, int ib, int g) {
  or_dom* d = &m->dom[ib];
  lview v;
  lev_dims(d, g, &v.n[0], &v.n[1], &v.n[2]);
  v.nj = v.n[1];
  v.nij = (int64_t)v.n[0] * v.n[1];
  v.nijk = d->faz[g] - v.nij * v.n[2];
  v.fi = d->cof;
  return v;
}

static int64_t lcell(const lview* v, int i, int j, int k) {
  return (int64_t)(k - 1) * v->nij + (int64_t)(i - 1) * v->nj + j + v->nijk;
}

/* A face plane of sync direction a (0: i, 1: j, 2: k) is addressed as
 * (c, u, w): c along the direction, (u, w) in the plane with u fastest in the
 * receive buffer, (w - 1) * ns1 + u: (j, k) for a = 0, (i, k) for a = 1,
 * (j, i) for a = 2 (exchangepp.for:69-122). */
static int64_t fcell(const lview* v, int a, int c, int u, int w) {
  if (a == 0) return lcell(v, c, u, w);
  if (a == 1) return lcell(v, u, c, w);
  return lcell(v, w, u, c);
}
static int fns1(const lview* v, int a) { return a == 1 ? v->n[0] : v->n[1]; }
static int fns2(const lview* v, int a) { return a == 2 ? v->n[0] : v->n[2]; }

/* Pack of sender sb's face plane for the receiver's buffer rb (prev: the
 * sender's first interior planes go to its previous neighbour).  Equal
 * resolution: the full plane (exchangepp.for:155-162); sender finer: the 8-cell
 * average of its two first planes on the receiver's coarse plane interior
 * (:164-174); sender coarser: 2 x its first plane on the four fine cells of
 * each coarse cell (:176-189). */
static void face_pack(const lview* s, int a, int prev, int cmp, double* rb) {
  const double* fi = s->fi;
  int ns1 = fns1(s, a), ns2 = fns2(s, a), na = s->n[a];
  if (cmp == 0) {
    int c = prev ? 2 : na - 1;
    for (int w = 1; w <= ns2; ++w)
      for (int u = 1; u <= ns1; ++u) rb[(w - 1) * ns1 + u] = fi[fcell(s, a, c, u, w)];
  } else if (cmp > 0) {
    int nsc1 = (ns1 - 2) / 2 + 2, nsc2 = (ns2 - 2) / 2 + 2;
    int c0 = prev ? 2 : na - 2;
    for (int w = 2; w <= nsc2 - 1; ++w)
      for (int u = 2; u <= nsc1 - 1; ++u) {
        int u0 = 2 * u - 2, w0 = 2 * w - 2;
        rb[(w - 1) * nsc1 + u] =
            0.125 * (fi[fcell(s, a, c0, u0, w0)] + fi[fcell(s, a, c0, u0 + 1, w0)] +
                     fi[fcell(s, a, c0, u0, w0 + 1)] + fi[fcell(s, a, c0, u0 + 1, w0 + 1)] +
                     fi[fcell(s, a, c0 + 1, u0, w0)] + fi[fcell(s, a, c0 + 1, u0 + 1, w0)] +
                     fi[fcell(s, a, c0 + 1, u0, w0 + 1)] + fi[fcell(s, a, c0 + 1, u0 + 1, w0 + 1)]);
      }
  } else {
    int nsr1 = 2 * (ns1 - 2) + 2;
    int c = prev ? 2 : na - 1;
    for (int w = 2; w <= ns2 - 1; ++w)
      for (int u = 2; u <= ns1 - 1; ++u) {
        double val = 2.0 * fi[fcell(s, a, c, u, w)];
        rb[(2 * w - 3) * nsr1 + 2 * u - 2] = val;
        rb[(2 * w - 3) * nsr1 + 2 * u - 1] = val;
        rb[(2 * w - 2) * nsr1 + 2 * u - 2] = val;
        rb[(2 * w - 2) * nsr1 + 2 * u - 1] = val;
      }
  }
}

/* Unpack into the receiver's ghost plane (prev: c = 1, next: c = n).  Equal:
 * the full plane (exchangepp.for:2106-2113); receiver finer: (r + 3 f1 - f2)/4
 * from the received value and its first two interior planes, over the full
 * plane (:2115-2123); receiver coarser: the plane's interior rows (:2125-2131). */
static void face_unpack(lview* r, int a, int prev, int cmp, const double* rb) {
  double* fi = r->fi;
  int ns1 = fns1(r, a), ns2 = fns2(r, a), na = r->n[a];
  int cg = prev ? 1 : na, c1 = prev ? 2 : na - 1, c2 = prev ? 3 : na - 2;
  if (cmp == 0) {
    for (int w = 1; w <= ns2; ++w)
      for (int u = 1; u <= ns1; ++u) fi[fcell(r, a, cg, u, w)] = rb[(w - 1) * ns1 + u];
  } else if (cmp > 0) {
    for (int w = 1; w <= ns2; ++w)
      for (int u = 1; u <= ns1; ++u)
        fi[fcell(r, a, cg, u, w)] =
            (rb[(w - 1) * ns1 + u] + 3.0 * fi[fcell(r, a, c1, u, w)] - fi[fcell(r, a, c2, u, w)]) / 4.0;
  } else {
    for (int w = 2; w <= ns2 - 1; ++w)
      for (int u = 2; u <= ns1 - 1; ++u) fi[fcell(r, a, cg, u, w)] = rb[(w - 1) * ns1 + u];
  }
}

/* Corner/edge sender cells: per axis (i, j, k) the code P2 ("2") or PN1
 * ("n-1"), or RUN for an edge's running index. */
static int lmr_pos(int code, int n, int run) { return code == RUN ? run : (code == P2 ? 2 : n - 1); }

/* The 8-cell average of a finer sender at a corner or edge: the 2x2x2 cells
 * from base (i0,j0,k0), summed with j, then i, then k as the fastest bit
 * (exchangepp.for:447-451, 653-659), divided by 8. */
static double avg8_jik(const lview* s, int i0, int j0, int k0) {
  const double* fi = s->fi;
  int64_t ll = lcell(s, i0, j0, k0), nj = s->nj, nij = s->nij;
  return (fi[ll] + fi[ll + 1] + fi[ll + nj] + fi[ll + 1 + nj] + fi[ll + nij] + fi[ll + 1 + nij] +
          fi[ll + nj + nij] + fi[ll + 1 + nj + nij]) / 8.0;
}

/* Trilinear value of a coarser sender at a fine corner/edge cell: 27, 9, 3, 1
 * weights of the cell and its neighbours toward the receiver (steps sj, si,
 * sk of +-1), in the j, i, k bit order, divided by 64 (exchangepp.for:452-458). */
static double interp64_jik(const lview* s, int i0, int j0, int k0, int si, int sj, int sk) {
  const double* fi = s->fi;
  int64_t ll = lcell(s, i0, j0, k0);
  int64_t dj = sj, di = (int64_t)si * s->nj, dk = (int64_t)sk * s->nij;
  return (27.0 * fi[ll] + 9.0 * fi[ll + dj] + 9.0 * fi[ll + di] + 3.0 * fi[ll + di + dj] + 9.0 * fi[ll + dk] +
          3.0 * fi[ll + dj + dk] + 3.0 * fi[ll + di + dk] + 1.0 * fi[ll + di + dj + dk]) / 64.0;
}

static int sgn_out(int code) { return code == P2 ? -1 : 1; }

/* A corner value for the receiver (exchangepp.for:441-640, 1400-1600). */
static double corner_pack(const lview* s, const int* code, int cmp) {
  if (cmp == 0) return s->fi[lcell(s, lmr_pos(code[0], s->n[0], 0), lmr_pos(code[1], s->n[1], 0),
                                   lmr_pos(code[2], s->n[2], 0))];
  if (cmp > 0) {
    int b[3];
    for (int a = 0; a < 3; ++a) b[a] = code[a] == P2 ? 2 : s->n[a] - 2;
    return avg8_jik(s, b[0], b[1], b[2]);
  }
  return interp64_jik(s, lmr_pos(code[0], s->n[0], 0), lmr_pos(code[1], s->n[1], 0),
                      lmr_pos(code[2], s->n[2], 0), sgn_out(code[0]), sgn_out(code[1]), sgn_out(code[2]));
}

/* An edge line for the receiver's buffer buf (exchangepp.for:646-1100,
 * 1604-2056): equal, nn = 2..len-1; sender finer, the averages of the fine
 * pairs 2nn-2, 2nn-1 on nn = 2..lenc-1; sender coarser, two fine values
 * 2nn-2 (running step -1) and 2nn-1 (+1) from each coarse cell. */
static void edge_pack(const lview* s, const int* code, int ax, int cmp, double* buf) {
  int len = s->n[ax];
  if (cmp == 0) {
    for (int nn = 2; nn <= len - 1; ++nn)
      buf[nn] = s->fi[lcell(s, lmr_pos(code[0], s->n[0], nn), lmr_pos(code[1], s->n[1], nn),
                            lmr_pos(code[2], s->n[2], nn))];
  } else if (cmp > 0) {
    int lenc = (len - 2) / 2 + 2;
    for (int nn = 2; nn <= lenc - 1; ++nn) {
      int b[3];
      for (int a = 0; a < 3; ++a) b[a] = code[a] == RUN ? 2 * nn - 2 : (code[a] == P2 ? 2 : s->n[a] - 2);
      buf[nn] = avg8_jik(s, b[0], b[1], b[2]);
    }
  } else {
    for (int nn = 2; nn <= len - 1; ++nn)
      for (int h = 0; h < 2; ++h) {
        int sg[3];
        for (int a = 0; a < 3; ++a) sg[a] = code[a] == RUN ? (h ? 1 : -1) : sgn_out(code[a]);
        buf[2 * nn - 2 + h] = interp64_jik(s, lmr_pos(code[0], s->n[0], nn), lmr_pos(code[1], s->n[1], nn),
                                           lmr_pos(code[2], s->n[2], nn), sg[0], sg[1], sg[2]);
      }
  }
}

static int rdv_cmp(const or_mg* m, int a, int b, int g) {
  int ra = RDV(m, a, g), rb = RDV(m, b, g);
  return ra == rb ? 0 : (ra > rb ? 1 : -1);
}

void or_exchangepp(or_mg* m, int g) { /* exchangepp.for:2-2835 */
  if (m->lmr)
    /* The reference reads receive-buffer entries no sender of this call wrote
     * (the ghost rows of a plane a coarser neighbour sends); they hold what an
     * earlier exchange left there.  Here they read as zero. */
    for (int ib = 0; ib < m->nbp; ++ib) {
      memset(m->dom[ib].recvb_m1, 0, sizeof(double) * ((size_t)m->ngg + 1));
      memset(m->dom[ib].recvb_p1, 0, sizeof(double) * ((size_t)m->ngg + 1));
    }
  for (int sync_dir = 1; sync_dir <= 3; ++sync_dir) {
    const int a = sync_dir - 1;
    /* pack loop, exchangepp.for:48-2063 (same-rank branches) */
    for (int ib = 0; ib < m->nbp; ++ib) {
      or_dom* d = &m->dom[ib];
      lview s = lview_of(m, ib, g);
      int cprev = d->d.nb_face[2 * a];
      int cnext = d->d.nb_face[2 * a + 1];
      if (cprev >= 0) face_pack(&s, a, 1, rdv_cmp(m, ib, cprev, g), m->dom[cprev].recvb_p1); /* :149-430 */
      if (sync_dir == 3) { /* prev corners and edges, :435-1100 */
        for (int c = 0; c < 4; ++c) {
          int nbr = d->d.nb_corner[c];
          if (nbr < 0) continue;
          m->dom[nbr].rc_p[c + 1] = corner_pack(&s, corprev_src[c], rdv_cmp(m, ib, nbr, g));
        }
        for (int e = 0; e < 6; ++e) {
          int nbr = d->d.nb_edge[e];
          if (nbr < 0) continue;
          edge_pack(&s, edgprev_src[e], edg_axis[e], rdv_cmp(m, ib, nbr, g), m->dom[nbr].re_p[e + 1]);
        }
      }
      if (cnext >= 0) face_pack(&s, a, 0, rdv_cmp(m, ib, cnext, g), m->dom[cnext].recvb_m1); /* :1107-1393 */
      if (sync_dir == 3) { /* next corners and edges, :1394-2060 */
        for (int c = 0; c < 4; ++c) {
          int nbr = d->d.nb_corner[4 + c];
          if (nbr < 0) continue;
          m->dom[nbr].rc_m[c + 1] = corner_pack(&s, cornext_src[c], rdv_cmp(m, ib, nbr, g));
        }
        for (int e = 0; e < 6; ++e) {
          int nbr = d->d.nb_edge[6 + e];
          if (nbr < 0) continue;
          edge_pack(&s, edgnext_src[e], edg_axis[e], rdv_cmp(m, ib, nbr, g), m->dom[nbr].re_m[e + 1]);
        }
      }
    }
    /* unpack loop, exchangepp.for:2066-2826 */
    for (int ib = 0; ib < m->nbp; ++ib) {
      or_dom* d = &m->dom[ib];
      lview r = lview_of(m, ib, g);
      int64_t nij = r.nij, nj = r.nj, nijk = r.nijk;
      double* fi = r.fi;
      int ni = r.n[0], nk = r.n[2];
      int cprev = d->d.nb_face[2 * a];
      int cnext = d->d.nb_face[2 * a + 1];
      if (cprev >= 0) face_unpack(&r, a, 1, rdv_cmp(m, ib, cprev, g), d->recvb_m1); /* :2101-2302 */
      if (cnext >= 0) face_unpack(&r, a, 0, rdv_cmp(m, ib, cnext, g), d->recvb_p1); /* :2306-2505 */
      if (sync_dir == 3) { /* :2511-2826, plain copies at every resolution */
        for (int c = 0; c < 4; ++c)
          if (d->d.nb_corner[c] >= 0)
            fi[PHI(pos(corprev_dst[c][0], ni, 0), pos(corprev_dst[c][1], nj, 0),
                   pos(corprev_dst[c][2], nk, 0))] = d->rc_m[c + 1];
        for (int e = 0; e < 6; ++e)
          if (d->d.nb_edge[e] >= 0) {
            int len = edge_len(e, ni, nj, nk);
            for (int nn = 2; nn <= len - 1; ++nn)
              fi[PHI(pos(edgprev_dst[e][0], ni, nn), pos(edgprev_dst[e][1], nj, nn),
                     pos(edgprev_dst[e][2], nk, nn))] = d->re_m[e + 1][nn];
          }
        for (int c = 0; c < 4; ++c)
          if (d->d.nb_corner[4 + c] >= 0)
            fi[PHI(pos(cornext_dst[c][0], ni, 0), pos(cornext_dst[c][1], nj, 0),
                   pos(cornext_dst[c][2], nk, 0))] = d->rc_p[c + 1];
        for (int e = 0; e < 6; ++e)
          if (d->d.nb_edge[6 + e] >= 0) {
            int len = edge_len(e, ni, nj, nk);
            for (int nn = 2; nn <= len - 1; ++nn)
              fi[PHI(pos(edgnext_dst[e][0], ni, nn), pos(edgnext_dst[e][1], nj, nn),
                     pos(edgnext_dst[e][2], nk, nn))] = d->re_p[e + 1][nn];
          }
      }
    }
  }
  or_mgbound(m, g);                        /* :2830 */
  if (m->periodic) or_exchbc_mgpp(m, g);   /* :2832 */
}

/* ------------------------------------------------------------ exchbc_mgpp */
void or_exchbc_mgpp(or_mg* m, int g) { /* exchangepp.for:2837-3454 */
  for (int ax = 0; ax < 3; ++ax) {
    /* pack (and single-block wrap) loop */
    for (int ib = 0; ib < m->nbp; ++ib) {
      or_dom* d = &m->dom[ib];
      if (!(d->d.bc[2 * ax] == 5 || d->d.bc[2 * ax + 1] == 5)) continue;
      int ni, nj, nk;
      lev_dims(d, g, &ni, &nj, &nk);
      int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
      double* fi = d->cof;
      int prev = d->d.nb_face[2 * ax], next = d->d.nb_face[2 * ax + 1];
      if (prev < 0) {
        if (next < 0) {
          if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) fi[PHI(1, j, k)] = fi[PHI(ni - 1, j, k)]; }
          else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) fi[PHI(i, 1, k)] = fi[PHI(i, nj - 1, k)]; }
          else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) fi[PHI(i, j, 1)] = fi[PHI(i, j, nk - 1)]; }
        } else {
          int pc = d->d.nb_periodic[2 * ax];
          if (pc >= 0) {
            double* rb = m->dom[pc].recvb_p1;
            if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) rb[(k - 1) * nj + j] = fi[PHI(2, j, k)]; }
            else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) rb[(k - 1) * ni + i] = fi[PHI(i, 2, k)]; }
            else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) rb[(j - 1) * ni + i] = fi[PHI(i, j, 2)]; }
          }
        }
      }
      if (next < 0) {
        if (prev < 0) {
          if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) fi[PHI(ni, j, k)] = fi[PHI(2, j, k)]; }
          else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) fi[PHI(i, nj, k)] = fi[PHI(i, 2, k)]; }
          else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) fi[PHI(i, j, nk)] = fi[PHI(i, j, 2)]; }
        } else {
          int pc = d->d.nb_periodic[2 * ax + 1];
          if (pc >= 0) {
            double* rb = m->dom[pc].recvb_m1;
            if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) rb[(k - 1) * nj + j] = fi[PHI(ni - 1, j, k)]; }
            else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) rb[(k - 1) * ni + i] = fi[PHI(i, nj - 1, k)]; }
            else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) rb[(j - 1) * ni + i] = fi[PHI(i, j, nk - 1)]; }
          }
        }
      }
    }
    /* unpack loop */
    for (int ib = 0; ib < m->nbp; ++ib) {
      or_dom* d = &m->dom[ib];
      if (!(d->d.bc[2 * ax] == 5 || d->d.bc[2 * ax + 1] == 5)) continue;
      int ni, nj, nk;
      lev_dims(d, g, &ni, &nj, &nk);
      int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
      double* fi = d->cof;
      int prev = d->d.nb_face[2 * ax], next = d->d.nb_face[2 * ax + 1];
      if (prev < 0 && next >= 0 && d->d.nb_periodic[2 * ax] >= 0) {
        const double* rb = d->recvb_m1;
        if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) fi[PHI(1, j, k)] = rb[(k - 1) * nj + j]; }
        else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) fi[PHI(i, 1, k)] = rb[(k - 1) * ni + i]; }
        else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) fi[PHI(i, j, 1)] = rb[(j - 1) * ni + i]; }
      }
      if (next < 0 && prev >= 0 && d->d.nb_periodic[2 * ax + 1] >= 0) {
        const double* rb = d->recvb_p1;
        if (ax == 0) { for (int k = 1; k <= nk; ++k) for (int j = 1; j <= nj; ++j) fi[PHI(ni, j, k)] = rb[(k - 1) * nj + j]; }
        else if (ax == 1) { for (int k = 1; k <= nk; ++k) for (int i = 1; i <= ni; ++i) fi[PHI(i, nj, k)] = rb[(k - 1) * ni + i]; }
        else { for (int j = 1; j <= nj; ++j) for (int i = 1; i <= ni; ++i) fi[PHI(i, j, nk)] = rb[(j - 1) * ni + i]; }
      }
    }
  }
}

/* ---------------------------------------------------------------- mgrelax */
static void relax_block_rbgs(or_dom* d, int g, int colour) {
  /* One colour pass of mgsolver.for:553-578 / :580-605.  Cells of one colour
   * do not read each other, so the pass is evaluated plane by plane in
   * storage order (j fastest, every second j); each cell's arithmetic is the
   * reference's. */
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
  int64_t nij2 = (int64_t)(ni - 2) * (nj - 2), incr = nij2 * (nk - 2);
  double* c = d->cof;
  int64_t faz = d->faz[g];
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
  for (int k = 2; k <= nk - 1; ++k)
    for (int i = 2; i <= ni - 1; ++i)
      for (int j = 2 + ((i + 2 + k + colour) & 1); j <= nj - 1; j += 2) {
        int64_t ijkphi = PHI(i, j, k);
        int64_t w = faz + (k - 2) * nij2 + (int64_t)(i - 2) * (nj - 2) + (j - 1);
        c[ijkphi] = (c[w + 7 * incr] -
                     (c[w] * c[ijkphi - nj] + c[w + incr] * c[ijkphi + nj] +
                      c[w + 2 * incr] * c[ijkphi - 1] + c[w + 3 * incr] * c[ijkphi + 1] +
                      c[w + 4 * incr] * c[ijkphi - nij] + c[w + 5 * incr] * c[ijkphi + nij])) /
                    c[w + 6 * incr];
      }
}

static void relax_block_lex(or_dom* d, int g) { /* mgsolver.for:407-432 */
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
  int64_t nij2 = (int64_t)(ni - 2) * (nj - 2), incr = nij2 * (nk - 2);
  double* c = d->cof;
  int64_t faz = d->faz[g];
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i) {
        int64_t ijkphi = PHI(i, j, k);
        int64_t w = faz + (k - 2) * nij2 + (int64_t)(i - 2) * (nj - 2) + (j - 1);
        c[ijkphi] = (c[w + 7 * incr] -
                     (c[w] * c[ijkphi - nj] + c[w + incr] * c[ijkphi + nj] +
                      c[w + 2 * incr] * c[ijkphi - 1] + c[w + 3 * incr] * c[ijkphi + 1] +
                      c[w + 4 * incr] * c[ijkphi - nij] + c[w + 5 * incr] * c[ijkphi + nij])) /
                    c[w + 6 * incr];
      }
}

static void relax_block_tdma(or_dom* d, int g, double* a, double* cc, int ngg) {
  /* mgsolver.for:434-549 */
  int ni, nj, nk;
  lev_dims(d, g, &ni, &nj, &nk);
  int64_t nij = (int64_t)ni * nj, nijk = d->faz[g] - (int64_t)ni * nj * nk;
  int64_t nij2 = (int64_t)(ni - 2) * (nj - 2), incr = nij2 * (nk - 2);
  double* c = d->cof;
  int64_t faz = d->faz[g];
  for (int q = 0; q <= ngg; ++q) { a[q] = 0.0; cc[q] = 0.0; }
#define WIDX(i, j, k) (faz + (int64_t)((k)-2) * nij2 + (int64_t)((i)-2) * (nj - 2) + ((j)-1))
  /* j-lines */
  for (int k = 2; k <= nk - 1; ++k)
    for (int i = 2; i <= ni - 1; ++i) {
      cc[1] = c[PHI(i, 1, k)];
      for (int j = 2; j <= nj - 1; ++j) {
        int64_t p = PHI(i, j, k), w = WIDX(i, j, k);
        double apr = 1.0 / (c[w + 6 * incr] - c[w + 2 * incr] * a[j - 1]);
        a[j] = c[w + 3 * incr] * apr;
        cc[j] = (c[w + 7 * incr] - c[w + incr] * c[p + nj] - c[w] * c[p - nj] -
                 c[w + 5 * incr] * c[p + nij] - c[w + 4 * incr] * c[p - nij] -
                 c[w + 2 * incr] * cc[j - 1]) * apr;
      }
      for (int j = nj - 1; j >= 2; --j) {
        int64_t p = PHI(i, j, k);
        c[p] = (cc[j] - a[j] * c[p + 1]);
      }
    }
  /* i-lines */
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 1; ++j) {
      cc[1] = c[PHI(1, j, k)];
      for (int i = 2; i <= ni - 1; ++i) {
        int64_t p = PHI(i, j, k), w = WIDX(i, j, k);
        double apr = 1.0 / (c[w + 6 * incr] - c[w] * a[i - 1]);
        a[i] = c[w + incr] * apr;
        cc[i] = (c[w + 7 * incr] - c[w + 3 * incr] * c[p + 1] - c[w + 2 * incr] * c[p - 1] -
                 c[w + 5 * incr] * c[p + nij] - c[w + 4 * incr] * c[p - nij] -
                 c[w] * cc[i - 1]) * apr;
      }
      for (int i = ni - 1; i >= 2; --i) {
        int64_t p = PHI(i, j, k);
        c[p] = (cc[i] - a[i] * c[p + nj]);
      }
    }
  /* k-lines */
  for (int i = 2; i <= ni - 1; ++i)
    for (int j = 2; j <= nj - 1; ++j) {
      cc[1] = c[PHI(i, j, 1)];
      for (int k = 2; k <= nk - 1; ++k) {
        int64_t p = PHI(i, j, k), w = WIDX(i, j, k);
        double apr = 1.0 / (c[w + 6 * incr] - c[w + 4 * incr] * a[k - 1]);
        a[k] = c[w + 5 * incr] * apr;
        cc[k] = (c[w + 7 * incr] - c[w + 3 * incr] * c[p + 1] - c[w + 2 * incr] * c[p - 1] -
                 c[w + incr] * c[p + nj] - c[w] * c[p - nj] - c[w + 4 * incr] * cc[k - 1]) * apr;
      }
      for (int k = nk - 1; k >= 2; --k) {
        int64_t p = PHI(i, j, k);
        c[p] = (cc[k] - a[k] * c[p + nij]);
      }
    }
#undef WIDX
}

void or_mgrelax(or_mg* m, int g, int it) { /* mgsolver.for:374-621 */
  double* a = NULL;
  double* cc = NULL;
  if (m->mg_itrsch == 2) {
    a = (double*)calloc((size_t)m->ngg + 1, sizeof(double));
    cc = (double*)calloc((size_t)m->ngg + 1, sizeof(double));
  }
  for (int itr = 1; itr <= it; ++itr) {
    for (int ib = 0; ib < m->nbp; ++ib) {
      or_dom* d = &m->dom[ib];
      if (m->mg_itrsch == 1) {
        relax_block_lex(d, g);
      } else if (m->mg_itrsch == 2) {
        relax_block_tdma(d, g, a, cc, m->ngg);
      } else {
        relax_block_rbgs(d, g, 0); /* MOD(i+j+k,2)==0, :553-578 */
        relax_block_rbgs(d, g, 1); /* MOD(i+j+k,2)==1, :580-605 */
      }
    }
    or_mgbound(m, g);     /* :614 */
    or_exchangepp(m, g);  /* :615 */
  }
  free(a);
  free(cc);
}

/* ---------------------------------------------------------------- mgrestr */
void or_mgrestr(or_mg* m, int glevel) { /* mgsolver.for:623-766 */
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    int nic, njc, nkc;
    lev_dims(d, glevel, &nic, &njc, &nkc);
    int64_t nijc2 = (int64_t)(nic - 2) * (njc - 2);
    int64_t incr_c = nijc2 * (nkc - 2);
    {
      int64_t base = d->faz[glevel] - (int64_t)nic * njc * nkc;
      memset(d->cof + base + 1, 0, sizeof(double) * (size_t)nic * njc * nkc);       /* :655-662 */
      memset(d->cof + d->faz[glevel] + 1 + 7 * incr_c, 0, sizeof(double) * (size_t)incr_c); /* :664-672 */
    }
    int nif, njf, nkf;
    int clamp = glevel > d->ngrid;
    if (clamp) { nif = nic; njf = njc; nkf = nkc; }
    else {
      int gl = glevel;
      nif = d->d.n[0] / ipow2(gl - 2) + 2;
      njf = d->d.n[1] / ipow2(gl - 2) + 2;
      nkf = d->d.n[2] / ipow2(gl - 2) + 2;
    }
    int64_t nij = (int64_t)nif * njf, nj = njf;
    int64_t nijk = d->faz[glevel - 1] - (int64_t)nif * njf * nkf;
    int64_t nijf2 = (int64_t)(nif - 2) * (njf - 2), incr_f = nijf2 * (nkf - 2);
    /* resf(nif,njf,nkf), Fortran column-major: (i,j,k) -> i-1 + nif*(j-1 + njf*(k-1)) */
    double* resf = (double*)calloc((size_t)nif * njf * nkf, sizeof(double));
#define RESF(i, j, k) resf[((int64_t)((k)-1) * njf + ((j)-1)) * nif + ((i)-1)]
    const double* c = d->cof;
    int64_t fazf = d->faz[glevel - 1];
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
    for (int k = 2; k <= nkf - 1; ++k)
      for (int i = 2; i <= nif - 1; ++i)
        for (int j = 2; j <= njf - 1; ++j) {
          int64_t p = PHI(i, j, k);
          int64_t w = fazf + (k - 2) * nijf2 + (int64_t)(i - 2) * (njf - 2) + (j - 1);
          RESF(i, j, k) = c[w + 7 * incr_f] -
                          (c[w] * c[p - njf] + c[w + incr_f] * c[p + njf] +
                           c[w + 2 * incr_f] * c[p - 1] + c[w + 3 * incr_f] * c[p + 1] +
                           c[w + 4 * incr_f] * c[p - nij] + c[w + 5 * incr_f] * c[p + nij] +
                           c[w + 6 * incr_f] * c[p]);
        }
    double* cw = d->cof;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
    for (int k = 2; k <= nkc - 1; ++k)
      for (int i = 2; i <= nic - 1; ++i)
        for (int j = 2; j <= njc - 1; ++j) {
          int64_t su = d->faz[glevel] + (k - 2) * nijc2 + (int64_t)(i - 2) * (njc - 2) + (j - 1) + 7 * incr_c;
          if (clamp) {
            cw[su] = RESF(i, j, k); /* :724-737 */
          } else { /* :741-756 */
            cw[su] = 0.125 * (RESF(2 * i - 2, 2 * j - 2, 2 * k - 2) + RESF(2 * i - 1, 2 * j - 2, 2 * k - 2) +
                              RESF(2 * i - 2, 2 * j - 1, 2 * k - 2) + RESF(2 * i - 1, 2 * j - 1, 2 * k - 2) +
                              RESF(2 * i - 2, 2 * j - 2, 2 * k - 1) + RESF(2 * i - 1, 2 * j - 2, 2 * k - 1) +
                              RESF(2 * i - 2, 2 * j - 1, 2 * k - 1) + RESF(2 * i - 1, 2 * j - 1, 2 * k - 1));
          }
        }
#undef RESF
    free(resf);
  }
}

/* ----------------------------------------------------------------- mgcorr */
void or_mgcorr(or_mg* m, int glevel) { /* mgsolver.for:768-910 */
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    int nif, njf, nkf;
    lev_dims(d, glevel, &nif, &njf, &nkf);
    int64_t nijf = (int64_t)nif * njf, nijkf = (int64_t)nif * njf * nkf;
    int nic, njc, nkc;
    int clamp = glevel >= d->ngrid;
    if (clamp) { nic = nif; njc = njf; nkc = nkf; }
    else {
      int gl = glevel;
      nic = d->d.n[0] / ipow2(gl) + 2;
      njc = d->d.n[1] / ipow2(gl) + 2;
      nkc = d->d.n[2] / ipow2(gl) + 2;
    }
    int64_t nijc = (int64_t)nic * njc, nijkc = (int64_t)nic * njc * nkc;
    double* c = d->cof;
    int64_t fazc = d->faz[glevel + 1], fazf = d->faz[glevel];
    if (clamp) { /* :812-824 */
      for (int kc = 1; kc <= nkc; ++kc)
        for (int ic = 1; ic <= nic; ++ic)
          for (int jc = 1; jc <= njc; ++jc) {
            int64_t ijkc = (kc - 1) * nijc + (int64_t)(ic - 1) * njc + jc + fazc - nijkc;
            int64_t ijkf = (kc - 1) * nijf + (int64_t)(ic - 1) * njf + jc + fazf - nijkf;
            c[ijkf] = c[ijkf] + c[ijkc];
          }
    } else { /* :828-896 */
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
      for (int kc = 1; kc <= nkc - 1; ++kc) {
        int k = 2 * kc - 1;
        for (int ic = 1; ic <= nic - 1; ++ic) {
          int i = 2 * ic - 1;
          for (int jc = 1; jc <= njc - 1; ++jc) {
            int j = 2 * jc - 1;
            int64_t q = (kc - 1) * nijc + (int64_t)(ic - 1) * njc + jc + fazc - nijkc;
            int64_t f = (int64_t)(k - 1) * nijf + (int64_t)(i - 1) * njf + j + fazf - nijkf;
            double c0 = c[q], cj = c[q + 1], ck = c[q + nijc], cjk = c[q + nijc + 1];
            double ci = c[q + njc], cij = c[q + njc + 1], cik = c[q + njc + nijc],
                   cijk = c[q + 1 + njc + nijc];
            c[f] = c[f] + (27.0 * c0 + 9.0 * cj + 9.0 * ck + 3.0 * cjk + 9.0 * ci + 3.0 * cij +
                           3.0 * cik + 1.0 * cijk) / 64.0;
            c[f + njf] = c[f + njf] + (9.0 * c0 + 3.0 * cj + 3.0 * ck + 1.0 * cjk + 27.0 * ci +
                                       9.0 * cij + 9.0 * cik + 3.0 * cijk) / 64.0;
            c[f + 1] = c[f + 1] + (9.0 * c0 + 27.0 * cj + 3.0 * ck + 9.0 * cjk + 3.0 * ci +
                                   9.0 * cij + 1.0 * cik + 3.0 * cijk) / 64.0;
            c[f + nijf] = c[f + nijf] + (9.0 * c0 + 3.0 * cj + 27.0 * ck + 9.0 * cjk + 3.0 * ci +
                                         1.0 * cij + 9.0 * cik + 3.0 * cijk) / 64.0;
            c[f + njf + 1] = c[f + njf + 1] + (3.0 * c0 + 9.0 * cj + 1.0 * ck + 3.0 * cjk +
                                               9.0 * ci + 27.0 * cij + 3.0 * cik + 9.0 * cijk) / 64.0;
            c[f + nijf + njf] = c[f + nijf + njf] + (3.0 * c0 + 1.0 * cj + 9.0 * ck + 3.0 * cjk +
                                                     9.0 * ci + 3.0 * cij + 27.0 * cik + 9.0 * cijk) / 64.0;
            c[f + nijf + 1] = c[f + nijf + 1] + (3.0 * c0 + 9.0 * cj + 9.0 * ck + 27.0 * cjk +
                                                 1.0 * ci + 3.0 * cij + 3.0 * cik + 9.0 * cijk) / 64.0;
            c[f + nijf + njf + 1] = c[f + nijf + njf + 1] + (1.0 * c0 + 3.0 * cj + 3.0 * ck + 9.0 * cjk +
                                                             3.0 * ci + 9.0 * cij + 9.0 * cik + 27.0 * cijk) / 64.0;
          }
        }
      }
    }
  }
  or_mgbound(m, glevel); /* :907 */
}

/* ----------------------------------------------------------------- mgkcyc */
void or_vcycle(or_mg* m) { /* mgsolver.for:272-352 */
  int L = m->ngrd_gl;
  int kount[MAXLEV + 2];
  int glevel = 1, kcycle = 1, nrel;
  or_mgrelax(m, 1, m->irestr);
  if (L == 1) goto post;
  or_mgrestr(m, glevel + 1);
  for (int l = 1; l <= L; ++l) kount[l] = 0;
  glevel = glevel + 1;
  nrel = m->irestr;
  for (;;) {
    if (glevel == 1) goto post;
    kount[glevel] = kount[glevel] + 1;
    or_mgrelax(m, glevel, nrel);
    if (kount[glevel] == kcycle + 1) {
      or_mgcorr(m, glevel - 1);
      kount[glevel] = 0;
      glevel = glevel - 1;
      nrel = m->iproln;
    } else if (glevel < L) {
      or_mgrestr(m, glevel + 1);
      glevel = glevel + 1;
      nrel = m->irestr;
    } else {
      or_mgrelax(m, glevel, m->iproln);
      or_mgcorr(m, glevel - 1);
      nrel = m->iproln;
      glevel = L - 1;
    }
  }
post:
  or_mgrelax(m, 1, m->iproln);
}

void or_mgkcyc(or_mg* m, double* const* pp, const double* const* su) {
  for (int ib = 0; ib < m->nbp; ++ib) { /* :239-266 */
    or_put_phi(m, 1, ib, pp[ib]);
    or_put_rhs(m, 1, ib, su[ib]);
  }
  or_vcycle(m);
  for (int ib = 0; ib < m->nbp; ++ib) or_get_phi(m, 1, ib, pp[ib]); /* :354-367 */
}

/* -------------------------------------------------------- outer iteration */
double or_residual(or_mg* m, double* const* p, const double* const* b,
                   double* const* r, double* bnorm2, double* rinf) {
  /* p's ghosts: the level-1 exchangepp (faces, then mgbound == pbound,
   * press.for:146-207) gives every face ghost the value exchange(4) gives;
   * edge/corner ghosts do not enter the 7-point operator. */
  for (int ib = 0; ib < m->nbp; ++ib) or_put_phi(m, 1, ib, p[ib]);
  or_exchangepp(m, 1);
  double rr = 0.0, bb = 0.0, rmax = 0.0;
  for (int ib = 0; ib < m->nbp; ++ib) {
    or_dom* d = &m->dom[ib];
    or_get_phi(m, 1, ib, p[ib]);
    int ni, nj, nk;
    lev_dims(d, 1, &ni, &nj, &nk);
    int64_t nij = (int64_t)ni * nj, nijk = d->faz[1] - (int64_t)ni * nj * nk;
    int64_t nij2 = (int64_t)(ni - 2) * (nj - 2), incr = nij2 * (nk - 2);
    const double* c = d->cof;
    double dv = d->d.h[0] * d->d.h[1] * d->d.h[2];
    /* per-plane partial sums, added in plane order: the result does not
     * depend on the thread count */
    double* part = (double*)calloc((size_t)3 * nk, sizeof(double));
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
    for (int k = 2; k <= nk - 1; ++k) {
      double brr = 0.0, bbb = 0.0, bmax = 0.0;
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 1; ++i) {
          int64_t ph = PHI(i, j, k);
          int64_t w = d->faz[1] + (k - 2) * nij2 + (int64_t)(i - 2) * (nj - 2) + (j - 1);
          int64_t q = ((int64_t)(k - 2) * (nj - 2) + (j - 2)) * (ni - 2) + (i - 2);
          double bv = b[ib][q];
          double rv = bv - (c[w] * c[ph - nj] + c[w + incr] * c[ph + nj] + c[w + 2 * incr] * c[ph - 1] +
                            c[w + 3 * incr] * c[ph + 1] + c[w + 4 * incr] * c[ph - nij] +
                            c[w + 5 * incr] * c[ph + nij] + c[w + 6 * incr] * c[ph]);
          if (r) r[ib][q] = rv;
          brr += rv * rv;
          bbb += bv * bv;
          double a = fabs(rv) * dv;
          if (!(a <= bmax)) bmax = a; /* keeps a NaN */
        }
      part[3 * k - 3] = brr;
      part[3 * k - 2] = bbb;
      part[3 * k - 1] = bmax;
    }
    for (int k = 2; k <= nk - 1; ++k) {
      rr += part[3 * k - 3];
      bb += part[3 * k - 2];
      if (!(part[3 * k - 1] <= rmax)) rmax = part[3 * k - 1];
    }
    free(part);
  }
  if (bnorm2) *bnorm2 = bb;
  if (rinf) *rinf = rmax;
  return rr;
}

int or_solve(or_mg* m, double* const* p, const double* const* b, double tol,
             int maxcy, int stop_rule, int* cycles, double* relres,
             double* history) {
  /* newsolv_mg.for:17-57: the outer loop is defect correction.  Each
   * iteration runs one V-cycle on pp from zero with the current defect as
   * right-hand side, then p += pp and the defect is recomputed in FP64. */
  int nb = m->nbp;
  double** r = (double**)calloc((size_t)nb, sizeof(double*));
  double** pp = (double**)calloc((size_t)nb, sizeof(double*));
  for (int ib = 0; ib < nb; ++ib) {
    const or_dom* d = &m->dom[ib];
    size_t ni = (size_t)d->d.n[0], nj = (size_t)d->d.n[1], nk = (size_t)d->d.n[2];
    r[ib] = (double*)calloc(ni * nj * nk, sizeof(double));
    pp[ib] = (double*)calloc((ni + 2) * (nj + 2) * (nk + 2), sizeof(double));
  }
  double bb, rinf;
  double rr = or_residual(m, p, b, r, &bb, &rinf);
  double bn = sqrt(bb) > 0 ? sqrt(bb) : 1.0;
  double rel = sqrt(rr) / bn;
  if (history) history[0] = rel;
  int iter = 0, status = 1;
  if (stop_rule == 0 && rel <= tol) status = 0;
  while (status != 0 && iter < maxcy) {
    for (int ib = 0; ib < nb; ++ib) {
      const or_dom* d = &m->dom[ib];
      size_t n = (size_t)(d->d.n[0] + 2) * (d->d.n[1] + 2) * (d->d.n[2] + 2);
      memset(pp[ib], 0, n * sizeof(double)); /* newsolv_mg.for:20-22, :45 */
    }
    or_mgkcyc(m, pp, (const double* const*)r);
    ++iter;
    for (int ib = 0; ib < nb; ++ib) { /* p = p + (pp - ppref), ppref = 0, :39-49 */
      const or_dom* d = &m->dom[ib];
      size_t n = (size_t)(d->d.n[0] + 2) * (d->d.n[1] + 2) * (d->d.n[2] + 2);
      for (size_t q = 0; q < n; ++q) p[ib][q] = (p[ib][q] + (pp[ib][q] - 0.0));
    }
    rr = or_residual(m, p, b, r, NULL, &rinf);
    rel = sqrt(rr) / bn;
    if (history) history[iter] = rel;
    if (stop_rule == 0 && rel <= tol) status = 0;
    if (stop_rule == 1 && rinf < tol && iter > 1) status = 0; /* :57 */
    if (!isfinite(rel)) { status = 2; break; }
  }
  if (cycles) *cycles = iter;
  if (relres) *relres = rel;
  for (int ib = 0; ib < nb; ++ib) { free(r[ib]); free(pp[ib]); }
  free(r);
  free(pp);
  return status;
}

/* ------------------------------------------------------------- projection */
/* Canonical index of cell (x, y, z) of a level-1 block array (nz+2, ny+2,
 * nx+2), x fastest, one ghost layer. */
#define CAN(x, y, z) ((((int64_t)(z)) * (ny + 2) + (y)) * (nx + 2) + (x))

void or_calvel(or_mg* m, double* const* u, double* const* v, double* const* w,
               const double* const* us, const double* const* vs, const double* const* ws,
               const double* const* p, const double* const* dens, double dt, double alfapr) {
  /* press.for:77-144.  Update ranges isu..ieu etc. (localparameters.for:
   * 106-133, 186-192): every interior face except the last one of an axis
   * that ends in a physical wall (no neighbour, bc /= 5). */
  for (int ib = 0; ib < m->nbp; ++ib) {
    const or_dom* d = &m->dom[ib];
    const int nx = d->d.n[0], ny = d->d.n[1], nz = d->d.n[2];
    const double dx = d->d.h[0], dy = d->d.h[1], dz = d->d.h[2];
    const int ieu = nx - ((d->d.nb_face[1] < 0 && d->d.bc[1] != 5) ? 1 : 0);
    const int jev = ny - ((d->d.nb_face[3] < 0 && d->d.bc[3] != 5) ? 1 : 0);
    const int kew = nz - ((d->d.nb_face[5] < 0 && d->d.bc[5] != 5) ? 1 : 0);
    const double* P = p[ib];
    const double* D = m->lsm ? dens[ib] : NULL;
    for (int k = 1; k <= nz; ++k) /* :88-101 */
      for (int i = 1; i <= ieu; ++i)
        for (int j = 1; j <= ny; ++j) {
          int64_t q = CAN(i, j, k);
          if (m->lsm)
            u[ib][q] = (us[ib][q] - dt * alfapr * (P[q + 1] - P[q]) / dx / (0.5 * (D[q] + D[q + 1])));
          else
            u[ib][q] = (us[ib][q] - dt * alfapr * (P[q + 1] - P[q]) / dx);
        }
    const int64_t sx = nx + 2, sxy = (int64_t)(nx + 2) * (ny + 2);
    for (int k = 1; k <= nz; ++k) /* :104-118 */
      for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= jev; ++j) {
          int64_t q = CAN(i, j, k);
          if (m->lsm)
            v[ib][q] = (vs[ib][q] - dt * alfapr * (P[q + sx] - P[q]) / dy / (0.5 * (D[q] + D[q + sx])));
          else
            v[ib][q] = (vs[ib][q] - dt * alfapr * (P[q + sx] - P[q]) / dy);
        }
    for (int k = 1; k <= kew; ++k) /* :120-134 */
      for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
          int64_t q = CAN(i, j, k);
          if (m->lsm)
            w[ib][q] = (ws[ib][q] - dt * alfapr * (P[q + sxy] - P[q]) / dz / (0.5 * (D[q] + D[q + sxy])));
          else
            w[ib][q] = (ws[ib][q] - dt * alfapr * (P[q + sxy] - P[q]) / dz);
        }
  }
}

/* The source of the face ghosts of face f (0..5 = W,E,S,N,B,T) of block ib
 * in the velocity exchanges: the neighbour (exchange_smlvl), the periodic
 * partner or the block itself (exchange_bc), or -1 for a physical wall. */
static int vel_face_source(const or_mg* m, int ib, int f) {
  const or_block_desc* d = &m->dom[ib].d;
  if (d->nb_face[f] >= 0) return d->nb_face[f];
  if (d->bc[f] != 5) return -1;
  if (d->nb_face[f ^ 1] < 0) return ib; /* single block along the axis: own wrap */
  return d->nb_periodic[f];
}

void or_vel_exchange(or_mg* m, double* const* fld) {
  /* exchange(1..3) as calvel ends (press.for:140-142), equal resolution:
   * exchange_bc (exchange_bc.for:17-...) then exchange_smlvl (exchange.for:
   * 302-1650).  Face ghost layer 0 on the interior rows (the rows the
   * unpack loops kspr..kepr, jspr..jepr cover, exchange.for:1560-1640):
   * a low-side ghost (x = 0) takes the source's last interior plane
   * (ie - ly with ie = its iep, x = nx), a high-side ghost (x = nx+1) the
   * source's first (is + ly, x = 1).  Physical walls keep their values.
   * Every written cell reads an interior cell, so the order is free. */
  for (int ib = 0; ib < m->nbp; ++ib) {
    const or_dom* d = &m->dom[ib];
    const int nx = d->d.n[0], ny = d->d.n[1], nz = d->d.n[2];
    for (int f = 0; f < 6; ++f) {
      const int s = vel_face_source(m, ib, f);
      if (s < 0) continue;
      const or_dom* S = &m->dom[s];
      const int sx_ = S->d.n[0], sy_ = S->d.n[1], sz_ = S->d.n[2];
      const int ax = f / 2, hi = f & 1;
      const double* src = fld[s];
      double* dst = fld[ib];
      for (int k = 1; k <= (ax == 2 ? 1 : nz); ++k)
        for (int j = 1; j <= (ax == 1 ? 1 : ny); ++j)
          for (int i = 1; i <= (ax == 0 ? 1 : nx); ++i) {
            int x = i, y = j, z = k, xs = i, ys = j, zs = k;
            if (ax == 0) { x = hi ? nx + 1 : 0; xs = hi ? 1 : sx_; }
            if (ax == 1) { y = hi ? ny + 1 : 0; ys = hi ? 1 : sy_; }
            if (ax == 2) { z = hi ? nz + 1 : 0; zs = hi ? 1 : sz_; }
            int64_t qs = (((int64_t)zs) * (sy_ + 2) + ys) * (sx_ + 2) + xs;
            dst[CAN(x, y, z)] = src[qs];
          }
    }
  }
}

double or_calmas(or_mg* m, const double* const* u, const double* const* v, const double* const* w,
                 double dt, double* const* su, double* rmax) {
  /* press.for:2-75, second-order branch (:40-62): fact = div u; su = fact/dt
   * (L_LSM: sup = fact*dx*dy*dz/dt); rmax = max |fact*dx*dy*dz|.  Returns
   * the sum of su^2 (per-plane partial sums added in plane order). */
  double ss = 0.0, rm = 0.0;
  for (int ib = 0; ib < m->nbp; ++ib) {
    const or_dom* d = &m->dom[ib];
    const int nx = d->d.n[0], ny = d->d.n[1], nz = d->d.n[2];
    const double dx = d->d.h[0], dy = d->d.h[1], dz = d->d.h[2];
    const int64_t sx = nx + 2, sxy = (int64_t)(nx + 2) * (ny + 2);
    double* part = (double*)calloc((size_t)2 * nz, sizeof(double));
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
    for (int k = 1; k <= nz; ++k) {
      double s2 = 0.0, mx = 0.0;
      for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
          int64_t q = CAN(i, j, k);
          double fact = ((u[ib][q] - u[ib][q - 1]) / dx + (v[ib][q] - v[ib][q - sx]) / dy +
                         (w[ib][q] - w[ib][q - sxy]) / dz);
          double r = m->lsm ? fact * dx * dy * dz / dt : fact / dt;
          su[ib][((int64_t)(k - 1) * ny + (j - 1)) * nx + (i - 1)] = r;
          s2 += r * r;
          double fact1 = fact * dx * dy * dz;
          double a = fabs(fact1);
          if (!(a <= mx)) mx = a; /* keeps a NaN */
        }
      part[2 * k - 2] = s2;
      part[2 * k - 1] = mx;
    }
    for (int k = 1; k <= nz; ++k) {
      ss += part[2 * k - 2];
      if (!(part[2 * k - 1] <= rm)) rm = part[2 * k - 1];
    }
    free(part);
  }
  if (rmax) *rmax = rm;
  return ss;
}

int or_project(or_mg* m, double* const* p, double* const* u, double* const* v, double* const* w,
               const double* const* us, const double* const* vs, const double* const* ws,
               const double* const* dens, double dt, double alfapr, double tol, int maxcy,
               int stop_rule, int* cycles, double* relres, double* rmax_out, double* history) {
  /* newsolv_mg.for:2-93 with the velocities: calvel, calmas, then per
   * iteration mgkcyc on pp = 0 with rhs su (sup for L_LSM), p = p + (pp -
   * ppref) over the block and its ghost layer, exchange(4) + pbound, calvel,
   * calmas.  stop_rule 1: rmax < tol .and. iter > 1 (:57); stop_rule 0:
   * ||su||2 <= tol * ||su||2 of the first calmas.  history (may be NULL)
   * receives maxcy+1 entries (rmax for rule 1, the relative norm for 0). */
  int nb = m->nbp;
  double** su = (double**)calloc((size_t)nb, sizeof(double*));
  double** pp = (double**)calloc((size_t)nb, sizeof(double*));
  for (int ib = 0; ib < nb; ++ib) {
    const or_dom* d = &m->dom[ib];
    size_t ni = (size_t)d->d.n[0], nj = (size_t)d->d.n[1], nk = (size_t)d->d.n[2];
    su[ib] = (double*)calloc(ni * nj * nk, sizeof(double));
    pp[ib] = (double*)calloc((ni + 2) * (nj + 2) * (nk + 2), sizeof(double));
  }
  double rmax;
  or_calvel(m, u, v, w, us, vs, ws, (const double* const*)p, dens, dt, alfapr); /* :16-17 */
  or_vel_exchange(m, u);
  or_vel_exchange(m, v);
  or_vel_exchange(m, w);
  double s0 = sqrt(or_calmas(m, (const double* const*)u, (const double* const*)v, (const double* const*)w, dt,
                             su, &rmax));
  double bn = s0 > 0 ? s0 : 1.0, rel = s0 / bn;
  if (history) history[0] = stop_rule == 1 ? rmax : rel;
  int iter = 0, status = 1;
  if (stop_rule == 0 && rel <= tol) status = 0;
  while (status != 0 && iter < maxcy) {
    for (int ib = 0; ib < nb; ++ib) {
      const or_dom* d = &m->dom[ib];
      size_t n = (size_t)(d->d.n[0] + 2) * (d->d.n[1] + 2) * (d->d.n[2] + 2);
      memset(pp[ib], 0, n * sizeof(double)); /* :20-22, :45 */
    }
    or_mgkcyc(m, pp, (const double* const*)su); /* :26 */
    ++iter;
    for (int ib = 0; ib < nb; ++ib) { /* :39-49, ppref = 0 */
      const or_dom* d = &m->dom[ib];
      size_t n = (size_t)(d->d.n[0] + 2) * (d->d.n[1] + 2) * (d->d.n[2] + 2);
      for (size_t q = 0; q < n; ++q) p[ib][q] = (p[ib][q] + (pp[ib][q] - 0.0));
    }
    /* exchange(4) + pbound (:51-52): the level-1 exchangepp gives every face
     * ghost the value they give (or_residual); edge and corner ghosts are
     * not read by calvel */
    for (int ib = 0; ib < nb; ++ib) or_put_phi(m, 1, ib, p[ib]);
    or_exchangepp(m, 1);
    for (int ib = 0; ib < nb; ++ib) or_get_phi(m, 1, ib, p[ib]);
    or_calvel(m, u, v, w, us, vs, ws, (const double* const*)p, dens, dt, alfapr); /* :54 */
    or_vel_exchange(m, u);
    or_vel_exchange(m, v);
    or_vel_exchange(m, w);
    double s = sqrt(or_calmas(m, (const double* const*)u, (const double* const*)v, (const double* const*)w, dt,
                              su, &rmax)); /* :55 */
    rel = s / bn;
    if (history) history[iter] = stop_rule == 1 ? rmax : rel;
    if (stop_rule == 0 && rel <= tol) status = 0;
    if (stop_rule == 1 && rmax < tol && iter > 1) status = 0; /* :57 */
    if (!isfinite(rel)) { status = 2; break; }
  }
  if (cycles) *cycles = iter;
  if (relres) *relres = rel;
  if (rmax_out) *rmax_out = rmax;
  for (int ib = 0; ib < nb; ++ib) { free(su[ib]); free(pp[ib]); }
  free(su);
  free(pp);
  return status;
}
#undef CAN

/* -------------------------------------------------------------------- SIP */
/* Stone's strongly implicit procedure on the pressure correction
 * (sipsol.for:2-205, ifi = 44) with the coefficients pressure_1sweep builds
 * (press.for:407-438: 1/dx^2, 1/dy^2, 1/dz^2, zero on the faces of physical
 * walls, ap = -(aw+ae+as+an+ab+at)).  pp is canonical with the ghost layer
 * (in/out), su interior.  The LU factors are rebuilt on every call, as the
 * reference does.  resab (may be NULL) receives sum |res| of every sweep;
 * returns the sweep count the reference leaves in nsweep. */
#define SIPC(x, y, z) ((((int64_t)(z)) * (ny + 2) + (y)) * (nx + 2) + (x))
typedef struct {
  double aw, ae, as, an, ab, at, ap;
} sip_coef;

static sip_coef sip_cell_coef(const or_block_desc* d, int x, int y, int z) {
  sip_coef c;
  const double dx = d->h[0], dy = d->h[1], dz = d->h[2];
  c.aw = 1.0 / (dx * dx);
  c.ae = 1.0 / (dx * dx);
  c.an = 1.0 / (dy * dy);
  c.as = 1.0 / (dy * dy);
  c.at = 1.0 / (dz * dz);
  c.ab = 1.0 / (dz * dz);
  if (d->nb_face[0] < 0 && d->bc[0] != 5 && x == 1) c.aw = 0.0;
  if (d->nb_face[1] < 0 && d->bc[1] != 5 && x == d->n[0]) c.ae = 0.0;
  if (d->nb_face[2] < 0 && d->bc[2] != 5 && y == 1) c.as = 0.0;
  if (d->nb_face[3] < 0 && d->bc[3] != 5 && y == d->n[1]) c.an = 0.0;
  if (d->nb_face[4] < 0 && d->bc[4] != 5 && z == 1) c.ab = 0.0;
  if (d->nb_face[5] < 0 && d->bc[5] != 5 && z == d->n[2]) c.at = 0.0;
  c.ap = -1.0 * (c.aw + c.ae + c.as + c.an + c.ab + c.at);
  return c;
}

int or_sipsol(or_mg* m, double* const* pp, const double* const* su, int nswp, double* resab_hist) {
  const double alfa = 0.92, small = 1e-20;
  const int nb = m->nbp;
  double** L = (double**)calloc((size_t)nb * 8, sizeof(double*));
  for (int ib = 0; ib < nb; ++ib) {
    const or_block_desc* d = &m->dom[ib].d;
    const size_t n = (size_t)(d->n[0] + 2) * (d->n[1] + 2) * (d->n[2] + 2);
    for (int q = 0; q < 8; ++q) L[8 * ib + q] = (double*)calloc(n, sizeof(double));
  }
  /* LU coefficients, sipsol.for:77-105 (loop order k, i, j) */
  for (int ib = 0; ib < nb; ++ib) {
    const or_block_desc* d = &m->dom[ib].d;
    const int nx = d->n[0], ny = d->n[1], nz = d->n[2];
    const int64_t sj = nx + 2, sk = (int64_t)(nx + 2) * (ny + 2);
    double *lb = L[8 * ib], *lw = L[8 * ib + 1], *ls = L[8 * ib + 2], *lpr = L[8 * ib + 3];
    double *un = L[8 * ib + 4], *ue = L[8 * ib + 5], *ut = L[8 * ib + 6];
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
          const int64_t q = SIPC(i, j, k);
          const sip_coef c = sip_cell_coef(d, i, j, k);
          /* ijk-nij = k-1, ijk-nj = i-1, ijk-1 = j-1 (the reference's j-fastest index) */
          lb[q] = c.ab / (1. + alfa * (un[q - sk] + ue[q - sk]));
          lw[q] = c.aw / (1. + alfa * (un[q - 1] + ut[q - 1]));
          ls[q] = c.as / (1. + alfa * (ue[q - sj] + ut[q - sj]));
          const double p1 = alfa * (lb[q] * un[q - sk] + lw[q] * un[q - 1]);
          const double p2 = alfa * (lb[q] * ue[q - sk] + ls[q] * ue[q - sj]);
          const double p3 = alfa * (lw[q] * ut[q - 1] + ls[q] * ut[q - sj]);
          lpr[q] = 1. / (c.ap + p1 + p2 + p3 - lb[q] * ut[q - sk] - lw[q] * ue[q - 1] - ls[q] * un[q - sj] + small);
          un[q] = (c.an - p1) * lpr[q];
          ue[q] = (c.ae - p2) * lpr[q];
          ut[q] = (c.at - p3) * lpr[q];
        }
  }
  double relast = 0.0, res1 = 0.0;
  int nsweep;
  for (nsweep = 1; nsweep <= nswp; ++nsweep) { /* :110-196 */
    double resab = 0.0;
    for (int ib = 0; ib < nb; ++ib) {
      const or_block_desc* d = &m->dom[ib].d;
      const int nx = d->n[0], ny = d->n[1], nz = d->n[2];
      const int64_t sj = nx + 2, sk = (int64_t)(nx + 2) * (ny + 2);
      double *lb = L[8 * ib], *lw = L[8 * ib + 1], *ls = L[8 * ib + 2], *lpr = L[8 * ib + 3];
      double *un = L[8 * ib + 4], *ue = L[8 * ib + 5], *ut = L[8 * ib + 6], *res = L[8 * ib + 7];
      double* fi = pp[ib];
      for (int k = 1; k <= nz; ++k) /* residual, :146-157 */
        for (int i = 1; i <= nx; ++i)
          for (int j = 1; j <= ny; ++j) {
            const int64_t q = SIPC(i, j, k);
            const sip_coef c = sip_cell_coef(d, i, j, k);
            const double s = su[ib][((int64_t)(k - 1) * ny + (j - 1)) * nx + (i - 1)];
            res[q] = (s - c.ap * fi[q] - c.an * fi[q + sj] - c.as * fi[q - sj] - c.ae * fi[q + 1] - c.aw * fi[q - 1] -
                      c.ab * fi[q - sk] - c.at * fi[q + sk]);
            resab = resab + fabs(res[q]);
          }
      for (int k = 1; k <= nz; ++k) /* forward substitution, :159-167 */
        for (int i = 1; i <= nx; ++i)
          for (int j = 1; j <= ny; ++j) {
            const int64_t q = SIPC(i, j, k);
            res[q] = (res[q] - lb[q] * res[q - sk] - lw[q] * res[q - 1] - ls[q] * res[q - sj]) * lpr[q];
          }
      for (int k = nz; k >= 1; --k) /* backward substitution and correction, :169-178 */
        for (int i = nx; i >= 1; --i)
          for (int j = ny; j >= 1; --j) {
            const int64_t q = SIPC(i, j, k);
            res[q] = res[q] - un[q] * res[q + sj] - ue[q] * res[q + 1] - ut[q] * res[q + sk];
            fi[q] = fi[q] + res[q];
          }
    }
    if (resab_hist) resab_hist[nsweep - 1] = resab;
    if (nsweep == 1) res1 = resab;
    const double rsm = resab / (res1 + small);
    or_vel_exchange(m, pp); /* exchange(44): face ghosts, walls untouched */
    const double reldif = fabs(rsm - relast); /* :187-192 */
    relast = rsm;
    if (rsm <= 0.001) break;
    if (reldif <= 0.00001) break;
  }
  if (nsweep > nswp) nsweep = nswp; /* :194 (the DO variable one past the end, minus one) */
  for (int q = 0; q < nb * 8; ++q) free(L[q]);
  free(L);
  return nsweep;
}
#undef SIPC

int or_pressure_1sweep(or_mg* m, double* const* p, double* const* u, double* const* v, double* const* w,
                       const double* const* us, const double* const* vs, const double* const* ws, double dt,
                       double alfapr, double eps, int niter, int nswp, int* iters, int* nsweeps, double* rmax_hist) {
  /* press.for:382-519 without the boundary updates after the loop: calvel,
   * then iterate calmas (stop on rmax < eps .and. iter > 1), sipsol(44) on
   * pp = 0, p = p + (pp - ppref), exchange(4) + pbound, calvel, at most niter
   * times.  rmax_hist (may be NULL) receives the rmax of every calmas (niter
   * entries at most).  Returns the last rmax. */
  const int nb = m->nbp;
  double** su = (double**)calloc((size_t)nb, sizeof(double*));
  double** pp = (double**)calloc((size_t)nb, sizeof(double*));
  for (int ib = 0; ib < nb; ++ib) {
    const or_dom* d = &m->dom[ib];
    size_t ni = (size_t)d->d.n[0], nj = (size_t)d->d.n[1], nk = (size_t)d->d.n[2];
    su[ib] = (double*)calloc(ni * nj * nk, sizeof(double));
    pp[ib] = (double*)calloc((ni + 2) * (nj + 2) * (nk + 2), sizeof(double));
  }
  double rmax = 0.0;
  int iter = 0, total = 0;
  or_calvel(m, u, v, w, us, vs, ws, (const double* const*)p, NULL, dt, alfapr);
  or_vel_exchange(m, u);
  or_vel_exchange(m, v);
  or_vel_exchange(m, w);
  for (;;) {
    iter = iter + 1;
    or_calmas(m, (const double* const*)u, (const double* const*)v, (const double* const*)w, dt, su, &rmax);
    if (rmax_hist) rmax_hist[iter - 1] = rmax;
    if (rmax < eps && iter > 1) break;
    total += or_sipsol(m, pp, (const double* const*)su, nswp, NULL);
    for (int ib = 0; ib < nb; ++ib) {
      const or_dom* d = &m->dom[ib];
      size_t n = (size_t)(d->d.n[0] + 2) * (d->d.n[1] + 2) * (d->d.n[2] + 2);
      for (size_t q = 0; q < n; ++q) {
        p[ib][q] = (p[ib][q] + (pp[ib][q] - 0.0));
        pp[ib][q] = 0.0;
      }
    }
    for (int ib = 0; ib < nb; ++ib) or_put_phi(m, 1, ib, p[ib]);
    or_exchangepp(m, 1);
    for (int ib = 0; ib < nb; ++ib) or_get_phi(m, 1, ib, p[ib]);
    or_calvel(m, u, v, w, us, vs, ws, (const double* const*)p, NULL, dt, alfapr);
    or_vel_exchange(m, u);
    or_vel_exchange(m, v);
    or_vel_exchange(m, w);
    if (!(iter < niter)) break;
  }
  if (iters) *iters = iter;
  if (nsweeps) *nsweeps = total;
  for (int ib = 0; ib < nb; ++ib) { free(su[ib]); free(pp[ib]); }
  free(su);
  free(pp);
  return 0;
}

/* --------------------------------------------------------------- topology */
int or_topology(int nblocks, const int32_t* ext, const int32_t* bc,
                or_block_desc* out) {
  /* read_infodom, alloc_dom.for:524-1200, on exact integer extents.
   * ext[6*b + (0..5)] = xs, xe, ys, ye, zs, ze. */
#define XS(b) ext[6 * (b) + 0]
#define XE(b) ext[6 * (b) + 1]
#define YS(b) ext[6 * (b) + 2]
#define YE(b) ext[6 * (b) + 3]
#define ZS(b) ext[6 * (b) + 4]
#define ZE(b) ext[6 * (b) + 5]
  int xst = XS(0), xen = XE(0), yst = YS(0), yen = YE(0), zst = ZS(0), zen = ZE(0);
  for (int b = 1; b < nblocks; ++b) {
    if (XS(b) < xst) xst = XS(b);
    if (XE(b) > xen) xen = XE(b);
    if (YS(b) < yst) yst = YS(b);
    if (YE(b) > yen) yen = YE(b);
    if (ZS(b) < zst) zst = ZS(b);
    if (ZE(b) > zen) zen = ZE(b);
  }
  for (int a = 0; a < nblocks; ++a) {
    or_block_desc* d = &out[a];
    d->n[0] = XE(a) - XS(a);
    d->n[1] = YE(a) - YS(a);
    d->n[2] = ZE(a) - ZS(a);
    d->origin[0] = XS(a);
    d->origin[1] = YS(a);
    d->origin[2] = ZS(a);
    for (int q = 0; q < 6; ++q) { d->bc[q] = bc[q]; d->nb_face[q] = -1; d->nb_periodic[q] = -1; }
    for (int q = 0; q < 8; ++q) d->nb_corner[q] = -1;
    for (int q = 0; q < 12; ++q) d->nb_edge[q] = -1;
    int say[6 + 8 + 12] = {0};
    for (int b = 0; b < nblocks; ++b) {
      if (b == a) continue;
      int sy = YS(a) == YS(b) && YE(a) == YE(b), sz = ZS(a) == ZS(b) && ZE(a) == ZE(b),
          sx = XS(a) == XS(b) && XE(a) == XE(b);
      /* faces, :545-680 */
      if (XS(a) == XE(b) && sy && sz) { d->nb_face[0] = b; say[0]++; }
      if (XE(a) == XS(b) && sy && sz) { d->nb_face[1] = b; say[1]++; }
      if (YS(a) == YE(b) && sx && sz) { d->nb_face[2] = b; say[2]++; }
      if (YE(a) == YS(b) && sx && sz) { d->nb_face[3] = b; say[3]++; }
      if (ZS(a) == ZE(b) && sx && sy) { d->nb_face[4] = b; say[4]++; }
      if (ZE(a) == ZS(b) && sx && sy) { d->nb_face[5] = b; say[5]++; }
      /* corners, :700-810 */
      if (XS(a) == XE(b) && YS(a) == YE(b) && ZS(a) == ZE(b)) { d->nb_corner[0] = b; say[6]++; }
      if (XS(a) == XE(b) && YE(a) == YS(b) && ZS(a) == ZE(b)) { d->nb_corner[1] = b; say[7]++; }
      if (XE(a) == XS(b) && YE(a) == YS(b) && ZS(a) == ZE(b)) { d->nb_corner[2] = b; say[8]++; }
      if (XE(a) == XS(b) && YS(a) == YE(b) && ZS(a) == ZE(b)) { d->nb_corner[3] = b; say[9]++; }
      if (XE(a) == XS(b) && YE(a) == YS(b) && ZE(a) == ZS(b)) { d->nb_corner[4] = b; say[10]++; }
      if (XE(a) == XS(b) && YS(a) == YE(b) && ZE(a) == ZS(b)) { d->nb_corner[5] = b; say[11]++; }
      if (XS(a) == XE(b) && YS(a) == YE(b) && ZE(a) == ZS(b)) { d->nb_corner[6] = b; say[12]++; }
      if (XS(a) == XE(b) && YE(a) == YS(b) && ZE(a) == ZS(b)) { d->nb_corner[7] = b; say[13]++; }
      /* edges, :824-1040 */
      if (XS(a) == XE(b) && ZS(a) == ZE(b) && sy) { d->nb_edge[0] = b; say[14]++; }
      if (YE(a) == YS(b) && ZS(a) == ZE(b) && sx) { d->nb_edge[1] = b; say[15]++; }
      if (XE(a) == XS(b) && ZS(a) == ZE(b) && sy) { d->nb_edge[2] = b; say[16]++; }
      if (YS(a) == YE(b) && ZS(a) == ZE(b) && sx) { d->nb_edge[3] = b; say[17]++; }
      if (XS(a) == XE(b) && YS(a) == YE(b) && sz) { d->nb_edge[4] = b; say[18]++; }
      if (XS(a) == XE(b) && YE(a) == YS(b) && sz) { d->nb_edge[5] = b; say[19]++; }
      if (XE(a) == XS(b) && ZE(a) == ZS(b) && sy) { d->nb_edge[6] = b; say[20]++; }
      if (YS(a) == YE(b) && ZE(a) == ZS(b) && sx) { d->nb_edge[7] = b; say[21]++; }
      if (XS(a) == XE(b) && ZE(a) == ZS(b) && sy) { d->nb_edge[8] = b; say[22]++; }
      if (YE(a) == YS(b) && ZE(a) == ZS(b) && sx) { d->nb_edge[9] = b; say[23]++; }
      if (XE(a) == XS(b) && YE(a) == YS(b) && sz) { d->nb_edge[10] = b; say[24]++; }
      if (XE(a) == XS(b) && YS(a) == YE(b) && sz) { d->nb_edge[11] = b; say[25]++; }
    }
    for (int q = 0; q < 26; ++q)
      if (say[q] > 1) return -1;
  }
  /* periodic partners, alloc_dom.for:1042-1200 */
  for (int a = 0; a < nblocks; ++a) {
    or_block_desc* d = &out[a];
    for (int b = 0; b < nblocks; ++b) {
      if (b == a) continue;
      int sy = YS(a) == YS(b) && YE(a) == YE(b), sz = ZS(a) == ZS(b) && ZE(a) == ZE(b),
          sx = XS(a) == XS(b) && XE(a) == XE(b);
      if (bc[0] == 5 && d->nb_face[0] < 0 && xen == XE(b) && sy && sz) d->nb_periodic[0] = b;
      if (bc[1] == 5 && d->nb_face[1] < 0 && xst == XS(b) && sy && sz) d->nb_periodic[1] = b;
      if (bc[2] == 5 && d->nb_face[2] < 0 && yen == YE(b) && sx && sz) d->nb_periodic[2] = b;
      if (bc[3] == 5 && d->nb_face[3] < 0 && yst == YS(b) && sx && sz) d->nb_periodic[3] = b;
      if (bc[4] == 5 && d->nb_face[4] < 0 && zen == ZE(b) && sx && sy) d->nb_periodic[4] = b;
      if (bc[5] == 5 && d->nb_face[5] < 0 && zst == ZS(b) && sx && sy) d->nb_periodic[5] = b;
    }
  }
  return 0;
#undef XS
#undef XE
#undef YS
#undef YE
#undef ZS
#undef ZE
}
