/*
 * h3d_oracle.h -- CPU oracle for the pressure-Poisson multigrid path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Hydro3D v7.0 multigrid routines, used by tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py as the checker.  It is never linked
 * into, loaded by, or called from the product library (hydro3d_b200).
 *
 * Parity pinning: the reference ships no golden vectors or known-answer
 * tests for this path and cannot be compiled here (Fortran and MPI; neither
 * toolchain is in the image).  The oracle is pinned by (a) golden fixtures
 * made by running the reference's own Fortran source (coeff, mgkcyc,
 * mgrelax, mgrestr, mgcorr, mgbound, exchangepp, exchbc_mgpp,
 * localparameters; calvel, calmas, pbound, exchange, exchange_smlvl,
 * exchange_bc) through the statement-by-statement translator in
 * oracle/fortran_ref.py (tests/golden/make_golden.py; the oracle reproduces
 * every fixture bit for bit, tests/test_golden.py), and (b) algebraic
 * properties (manufactured Neumann cosine modes, null space, symmetry).
 *
 * Every routine cites the reference file:line it restates.  Storage keeps the
 * reference's per-block `cof` work array and its j-fastest level layout
 * (mgsolver.for:62-66, 119-120), so lexicographic and line-TDMA orderings are
 * the reference's own.
 */
#ifndef H3D_ORACLE_H
#define H3D_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same byte layout as h3d_block_desc in include/h3d_mg.h (kept separate so
 * the oracle does not depend on the product headers). */
typedef struct {
  int32_t n[3];           /* interior cells i (x), j (y), k (z)              */
  int32_t ttc[3];         /* host dims incl. ghosts (unused by the oracle)   */
  int32_t pl;             /* host ghost width (unused by the oracle)         */
  int32_t ngrid;          /* levels of this block                             */
  double h[3];            /* dx, dy, dz                                       */
  int32_t nb_face[6];     /* iprev inext jprev jnext kprev knext              */
  int32_t nb_corner[8];   /* corprev1..4 cornext1..4                          */
  int32_t nb_edge[12];    /* edgprev1..6 edgnext1..6                          */
  int32_t nb_periodic[6]; /* per_ip per_in per_jp per_jn per_kp per_kn        */
  int32_t bc[6];          /* bc_west bc_east bc_south bc_north bc_bottom bc_top */
  int32_t rdiv;           /* local mesh refinement ratio (a power of 2; LMR)   */
  int32_t origin[3];      /* global cell index of the first interior cell     */
} or_block_desc;

typedef struct or_mg or_mg;

/* Create the solver state (localparameters.for:202-239 sizing). */
or_mg* or_create(int nblocks, const or_block_desc* blocks, int ngrd_gl,
                 int mg_itrsch, int irestr, int iproln, int lsm);
void or_destroy(or_mg* m);
int or_error(const or_mg* m); /* 0 if the configuration was accepted */

/* Interior density of block ib, x-fastest (n_z, n_y, n_x). LSM only. */
void or_set_density(or_mg* m, int ib, const double* dens);
/* coeff, mgsolver.for:2-224 */
void or_coeff(or_mg* m);

/* Level-g iterate of block ib, canonical x-fastest (nz+2, ny+2, nx+2) incl.
 * the one ghost layer; rhs is interior only (nz, ny, nx). */
void or_put_phi(or_mg* m, int g, int ib, const double* a);
void or_get_phi(const or_mg* m, int g, int ib, double* a);
void or_put_rhs(or_mg* m, int g, int ib, const double* a);
void or_get_rhs(const or_mg* m, int g, int ib, double* a);
/* Coefficient slot s (0 aw,1 ae,2 as,3 an,4 ab,5 at,6 ap) interior-only. */
void or_get_coef(const or_mg* m, int g, int ib, int s, double* a);

/* Scales the coefficient slots aw..ap of level g by s (not a reference
 * routine: models the product's consistent L_LSM coarse scaling). */
void or_scale_level_coef(or_mg* m, int g, double s);
/* Overwrites coefficient slot s of level g, block ib (interior, x fastest). */
void or_set_coef(or_mg* m, int g, int ib, int s, const double* a);

/* Reference subroutines on the resident state. */
void or_mgrelax(or_mg* m, int g, int it);   /* mgsolver.for:374-621 */
void or_mgrestr(or_mg* m, int g);           /* mgsolver.for:623-766 */
void or_mgcorr(or_mg* m, int g);            /* mgsolver.for:768-910 */
void or_mgbound(or_mg* m, int g);           /* mgsolver.for:912-997 */
void or_exchangepp(or_mg* m, int g);        /* exchangepp.for:2-2835 */
void or_exchbc_mgpp(or_mg* m, int g);       /* exchangepp.for:2837-3454 */
void or_vcycle(or_mg* m);                   /* mgkcyc control flow, mgsolver.for:272-352 */

/* mgkcyc on level-1 arrays: pp (canonical with ghosts) in/out, su interior. */
void or_mgkcyc(or_mg* m, double* const* pp, const double* const* su);

/* r = b - A p on level 1 (FP64), with p's face ghosts filled first the way
 * exchange(4)+pbound leave them.  p is canonical with ghosts (ghosts are
 * rewritten), b and r interior-only.  Returns sum r^2; *bnorm2 = sum b^2;
 * *rinf = max |r| * dV (the calmas rmax measure, press.for:61-63). */
double or_residual(or_mg* m, double* const* p, const double* const* b,
                   double* const* r, double* bnorm2, double* rinf);

/* newsolv_mg outer loop (newsolv_mg.for:17-57) written as defect correction
 * on b - A p.  stop_rule 0: ||r||2/||b||2 <= tol (checked before each cycle);
 * stop_rule 1: reference rule rmax < tol .and. iter > 1 (checked after each
 * cycle).  history (may be NULL) receives maxcy+1 relative residuals. */
int or_solve(or_mg* m, double* const* p, const double* const* b, double tol,
             int maxcy, int stop_rule, int* cycles, double* relres,
             double* history);

/* The projection (press.for:2-144, newsolv_mg.for:2-93).  Face velocities
 * use the canonical level-1 layout of the cell they belong to: u(x,y,z) is
 * the east face of cell (x,y,z), x = 0 the block's west face (a ghost), and
 * likewise v (north faces) and w (top faces).  dens (L_LSM only) is the
 * level-1 density, canonical with its face ghosts as the host's exchange
 * left them. */
void or_calvel(or_mg* m, double* const* u, double* const* v, double* const* w,
               const double* const* us, const double* const* vs, const double* const* ws,
               const double* const* p, const double* const* dens, double dt, double alfapr);
/* exchange(1..3) of one velocity component: face ghosts, interior rows. */
void or_vel_exchange(or_mg* m, double* const* fld);
/* calmas: su (interior, (nz,ny,nx)) and rmax; returns sum su^2. */
double or_calmas(or_mg* m, const double* const* u, const double* const* v, const double* const* w,
                 double dt, double* const* su, double* rmax);
/* newsolv_mg with the velocities.  Returns 0 converged, 1 not converged,
 * 2 diverged. */
int or_project(or_mg* m, double* const* p, double* const* u, double* const* v, double* const* w,
               const double* const* us, const double* const* vs, const double* const* ws,
               const double* const* dens, double dt, double alfapr, double tol, int maxcy,
               int stop_rule, int* cycles, double* relres, double* rmax, double* history);

/* Stone's SIP (sipsol.for:2-205, ifi = 44) on pp (canonical with ghosts,
 * in/out) with rhs su (interior) and pressure_1sweep's coefficients; at most
 * nswp sweeps; resab (may be NULL) receives sum |res| per sweep.  Returns the
 * reference's nsweep. */
int or_sipsol(or_mg* m, double* const* pp, const double* const* su, int nswp, double* resab);
/* pressure_1sweep (press.for:382-519) without its closing boundu/v/w: the
 * SIP pressure loop over the velocities.  rmax_hist (may be NULL, niter
 * entries) gets the rmax of every calmas. */
int or_pressure_1sweep(or_mg* m, double* const* p, double* const* u, double* const* v, double* const* w,
                       const double* const* us, const double* const* vs, const double* const* ws, double dt,
                       double alfapr, double eps, int niter, int nswp, int* iters, int* nsweeps,
                       double* rmax_hist);

/* Block topology from integer extents: read_infodom neighbour discovery
 * (alloc_dom.for:524-1200).  ext is nblocks x 6 (x0,x1,y0,y1,z0,z1) in global
 * cell units; bc[6] global codes.  Fills nb_face/nb_corner/nb_edge/
 * nb_periodic/bc/n/origin of each desc. Returns 0, or -1 on ambiguity. */
int or_topology(int nblocks, const int32_t* ext, const int32_t* bc,
                or_block_desc* out);

/* OpenMP thread count used by the colour passes (1 = scalar). */
void or_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
