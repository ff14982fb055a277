/*
 * h3d_mg.h -- C ABI of the B200 pressure-Poisson multigrid solver.
 *
 * Drop-in for Hydro3D v7.0's multigrid pressure path (src_v70/newsolv_mg.for,
 * src_v70/mgsolver.for, src_v70/exchangepp.for).  The Fortran host keeps its
 * `dom(ib)` block arrays and calls these entry points through an
 * ISO_C_BINDING interface; arrays are passed as the address of element
 * (1,1,1) of the Fortran array (i fastest), sizes as plain integers.
 *
 * Conventions
 *   - Every entry point returns H3D_OK (0) or a negative H3D_ERR_* code and
 *     never exits the process (the reference prints and STOPs:
 *     newsolv_mg.for:61-75, localparameters.for:204-208).
 *   - One handle = one GPU + one CUDA stream; calls on a handle are not
 *     re-entrant.  Device memory persists across calls.
 *   - "Host field" = a Fortran array dims ttc[0..2] with pl ghost layers
 *     (module_multidata.for:52-56: p, pp, su, sup, dens).
 *   - "Canonical level array" = float64 (nz+2, ny+2, nx+2), x fastest, one
 *     ghost layer, where n* is the block's interior size at that level;
 *     a canonical right-hand side is (nz, ny, nx).
 */
#ifndef H3D_MG_H
#define H3D_MG_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H3D_OK 0
#define H3D_ERR_BAD_CONFIG (-1)    /* sizes/levels/topology the path does not support */
#define H3D_ERR_CUDA (-2)          /* a CUDA runtime call failed */
#define H3D_ERR_NOT_CONVERGED (-3) /* maxcy reached ('not converged!!', newsolv_mg.for:61) */
#define H3D_ERR_DIVERGED (-4)      /* NaN/Inf or growth ('BIG RMAX', newsolv_mg.for:65-75) */
#define H3D_ERR_TIMEOUT (-5)       /* a bounded device wait gave up */
#define H3D_ERR_NO_DEVICE (-6)     /* no CUDA device / wrong architecture */
#define H3D_ERR_ARG (-7)           /* bad argument (null pointer, index out of range) */
#define H3D_ERR_OOM (-8)           /* device allocation failed */
#define H3D_ERR_INTERNAL (-9)

/* One block (`type multidom`, module_multidata.for:16-120). */
typedef struct h3d_block_desc {
  int32_t n[3];           /* interior cells iep-isp+1, jep-jsp+1, kep-ksp+1 */
  int32_t ttc[3];         /* host array dims ttc_i, ttc_j, ttc_k */
  int32_t pl;             /* host ghost width (localparameters.for:19-23) */
  int32_t ngrid;          /* dom(ib)%ngrid */
  double h[3];            /* dx, dy, dz */
  int32_t nb_face[6];     /* iprev inext jprev jnext kprev knext (-1 = none) */
  int32_t nb_corner[8];   /* corprev1..4, cornext1..4 */
  int32_t nb_edge[12];    /* edgprev1..6, edgnext1..6 */
  int32_t nb_periodic[6]; /* per_ip per_in per_jp per_jn per_kp per_kn */
  int32_t bc[6];          /* bc_west bc_east bc_south bc_north bc_bottom bc_top; 5 = periodic */
  int32_t rdiv;           /* local mesh refinement ratio rdiv (a power of 2, LMR = 2;
                             localparameters.for:24-59): n and h are the refined block's,
                             ngrid = ngrid_input + log2(rdiv) */
  int32_t origin[3];      /* global index of the first interior cell (informational) */
} h3d_block_desc;

#define H3D_PREC_FP64 0   /* plain FP64 V-cycle (reference arithmetic) */
#define H3D_PREC_MIXED 1  /* FP32 V-cycle inside FP64 iterative refinement */

typedef struct h3d_mg_desc {
  int32_t nblocks;
  int32_t ngrd_gl;        /* MG levels (module_vars.for:8) */
  int32_t mg_itrsch;      /* smoother (mgsolver.for:374-621): 1 lexicographic GS, 2 line TDMA,
                             3 red-black GS (the fast path; 1 and 2 run as wavefronts) */
  int32_t irestr, iproln; /* pre/post sweeps (control.cin line 11) */
  int32_t maxcy;          /* default cycle cap for h3d_mg_newsolv */
  int32_t precision;      /* H3D_PREC_* */
  int32_t var_coef;       /* 0: constant coefficients; 1: L_LSM density coefficients */
  int32_t device;         /* CUDA ordinal */
  int32_t coarse_sweeps;  /* sweeps at the coarsest level; 0 = irestr+iproln (reference) */
  int32_t inner_cycles;   /* MIXED: FP32 V-cycles per FP64 refinement step (0 = 2) */
  int32_t use_graph;      /* 1: capture each V-cycle as a CUDA graph */
  int32_t coarse_op;      /* L_LSM coarse levels: 0 = coeff's coefficients from the averaged
                             density (mgsolver.for:78-184, the reference); 1 = face-sum
                             coarsening (each coarse face = sum of its four fine faces / 16),
                             which keeps converging at 1000:1 density ratios */
  int32_t coarse_direct;  /* 1: with coarse_sweeps > 0, solve a small coarsest level (at most
                             512 cells, constant coefficients, symmetric) directly by its
                             pseudo-inverse instead of the sweeps; 0: the sweeps */
  int32_t rb_order;       /* MIXED, FP32 levels: 0 = the reference's order (a block's black
                             cells see the other blocks' red cells as they were before the
                             sweep, mgsolver.for:614-615); 1 = red-black order across block
                             faces (the red cells next to block faces are computed ahead of
                             the sweep; the coarse tail fills ghosts after each colour) */
  float omega;            /* MIXED, FP32 levels: over-relaxation factor of the red-black
                             sweeps, x + omega (gs - x); 0 = 1 (Gauss-Seidel); below 2 */
  const h3d_block_desc* blocks;
} h3d_mg_desc;

typedef struct h3d_mg h3d_mg;

/* Options and report of a solve. */
typedef struct h3d_solve_opts {
  double tol;             /* tolerance (see stop_rule) */
  int32_t maxcy;          /* cycle cap (0 = desc.maxcy) */
  int32_t stop_rule;      /* 0: ||b-Ap||2/||b||2 <= tol, checked before each cycle;
                             1: reference rule rmax < tol .and. iter > 1 (newsolv_mg.for:57);
                             2: every block's own ||b-Ap||2/||b||2 <= tol (independent
                                blocks; needs even nx in every block) */
  int32_t remove_mean;    /* 1: subtract the FP64 mean of p at the end (all-Neumann) */
  int32_t record_history; /* 1: keep ||r||/||b|| per cycle (read with h3d_mg_history) */
} h3d_solve_opts;

typedef struct h3d_solve_info {
  int32_t cycles;         /* V-cycles run (inner FP32 cycles for MIXED) */
  int32_t outer;          /* FP64 defect evaluations after the initial one */
  double relres;          /* final ||b-Ap||2/||b||2 (FP64) */
  double rmax;            /* final max|b-Ap| * dV (calmas measure, press.for:61-63) */
  double bnorm;           /* ||b||2 */
  double device_ms;       /* device time of the solve, CUDA events on the solve stream */
  double smoother_ms;     /* device time in the full level-1 sweeps (profiling on; the first
                             sweep from a zero iterate is not included) */
  int64_t smoother_launches;
  int64_t kernel_launches;/* kernels this library launched during the solve */
  double smoother_bytes;  /* algorithmic bytes of the profiled level-1 smoother launches */
  double relres_block_max;/* stop_rule 2: largest per-block ||b-Ap||2/||b||2; else = relres */
} h3d_solve_info;

/* --- set-up (localparameters.for:202-239, initial.for:329-360, coeff) ---- */
int h3d_mg_create(h3d_mg** out, const h3d_mg_desc* desc);
int h3d_mg_destroy(h3d_mg* h);
/* Density of block ib as a host field (ttc dims, pl ghosts); L_LSM only.
 * Replaces the dom(ib)%dens read in coeff (mgsolver.for:82); the first ghost
 * layer is kept for calvel's face densities (press.for:92-94). */
int h3d_mg_set_density(h3d_mg* h, int32_t ib, const double* dens);
/* coeff (mgsolver.for:2-224): per-level coefficients on the device. */
int h3d_mg_coeff(h3d_mg* h);

/* --- the drop-in calls -------------------------------------------------- */
/* mgkcyc (mgsolver.for:226-372): one V-cycle.  pp[ib] host field in/out
 * (interior + first ghost layer used), su[ib] host field (interior read). */
int h3d_mg_mgkcyc(h3d_mg* h, double* const* pp, const double* const* su);
/* newsolv_mg (newsolv_mg.for:17-57) as FP64 defect correction on b - A p.
 * p[ib] host field in/out, b[ib] host field (su, or sup for L_LSM). */
int h3d_mg_newsolv(h3d_mg* h, double* const* p, const double* const* b,
                   const h3d_solve_opts* opts, h3d_solve_info* info);

/* --- device-resident operation ------------------------------------------ */
#define H3D_FIELD_P 0     /* level-1 pressure, FP64, canonical with ghosts */
#define H3D_FIELD_B 1     /* level-1 right-hand side, FP64, canonical interior */
/* Face velocities of the projection, FP64, canonical with the ghost layer:
 * entry (x,y,z) of U is the east face of cell (x,y,z) (x = 0: the block's
 * west face), V north faces, W top faces; the host arrays are the reference's
 * dom(ib)%u, v, w (module_multidata.for:52) and ustar, vstar, wstar (:64-65). */
#define H3D_FIELD_U 2
#define H3D_FIELD_V 3
#define H3D_FIELD_W 4
#define H3D_FIELD_USTAR 5
#define H3D_FIELD_VSTAR 6
#define H3D_FIELD_WSTAR 7
/* The SIP pressure correction pp (sipsol.for), FP64, canonical with ghosts. */
#define H3D_FIELD_PP 8
/* Copy block ib of a resident field from/to a host field (ttc dims, pl ghosts). */
int h3d_mg_upload(h3d_mg* h, int32_t field, int32_t ib, const double* host);
int h3d_mg_download(h3d_mg* h, int32_t field, int32_t ib, double* host);
/* Zero a resident field on the device (e.g. the initial guess pp = 0,
 * newsolv_mg.for:20-22). */
int h3d_mg_zero_field(h3d_mg* h, int32_t field);
/* Solve with p and b already in device memory. */
int h3d_mg_solve_resident(h3d_mg* h, const h3d_solve_opts* opts, h3d_solve_info* info);
/* ||b-Ap||^2, ||b||^2 and max|b-Ap|*dV of the resident fields. */
int h3d_mg_residual(h3d_mg* h, double* rr, double* bb, double* rinf);
/* Relative residual history of the last solve (n <= cap entries written). */
int h3d_mg_history(h3d_mg* h, double* out, int32_t cap, int32_t* n);

/* --- the projection on resident fields (press.for, newsolv_mg.for) ------ */
/* calvel (press.for:77-144) with its exchange(1..3): U, V, W from USTAR,
 * VSTAR, WSTAR and the resident pressure, on the faces the reference updates
 * (every interior face but the last one before a physical wall,
 * localparameters.for:186-192), divided by the face density for L_LSM (the
 * density of h3d_mg_set_density, ghost layer included); then the face ghosts
 * of the interior rows from the neighbouring or periodic block.  Faces on
 * physical walls keep their values (the boundary condition). */
int h3d_mg_calvel(h3d_mg* h, double dt, double alfapr);
/* calmas (press.for:2-75, second-order branch): su = div u / dt (L_LSM:
 * sup = div u * dx*dy*dz / dt) into H3D_FIELD_B and the level-1 right-hand
 * side; *rmax = max |div u * dx*dy*dz| (:61-63), *su2 = sum su^2 (either may
 * be NULL). */
int h3d_mg_calmas(h3d_mg* h, double dt, double* rmax, double* su2);
/* exchange(4) + pbound (press.for:146-207) on the resident pressure: every
 * face ghost of the interior rows from the neighbour, periodic partner or
 * (physical wall) the adjacent interior cell. */
int h3d_mg_pbound(h3d_mg* h);
/* newsolv_mg (newsolv_mg.for:2-93) with the velocities: calvel, calmas, then
 * per iteration mgkcyc on pp = 0 with rhs su (MIXED: FP32 V-cycles), p = p +
 * pp over the block and its ghost layer, exchange(4) + pbound, calvel,
 * calmas.  stop_rule 1: the reference's rmax < tol .and. iter > 1 (:57);
 * stop_rule 0: ||su||2 <= tol * ||su||2 of the first calmas (info->bnorm);
 * stop_rule 2 is rejected.  info->rmax and info->relres report the last
 * calmas.  Reads P, U, V, W, USTAR, VSTAR, WSTAR; writes P, U, V, W, B.
 * Edge and corner ghosts of P keep p + pp (calvel does not read them). */
int h3d_mg_project_resident(h3d_mg* h, double dt, double alfapr, const h3d_solve_opts* opts,
                            h3d_solve_info* info);
/* The same from host fields (ttc dims, pl ghosts; the first ghost layer is
 * read and written): p, u, v, w in/out, ustar, vstar, wstar in. */
int h3d_mg_project(h3d_mg* h, double* const* p, double* const* u, double* const* v, double* const* w,
                   const double* const* ustar, const double* const* vstar, const double* const* wstar,
                   double dt, double alfapr, const h3d_solve_opts* opts, h3d_solve_info* info);

/* --- the SIP pressure path (solver = 1: press.for:382-519, sipsol.for) --- */
/* sipsol(44) (sipsol.for:2-205): Stone's strongly implicit procedure on the
 * resident correction H3D_FIELD_PP with right-hand side H3D_FIELD_B and the
 * coefficients pressure_1sweep builds (press.for:407-438); LU factors
 * rebuilt on every call as the reference does; at most nswp sweeps, each
 * followed by exchange(44) (face ghosts from neighbours and periodic
 * partners), stopping when sum |res| falls to 0.001 of the first sweep's or
 * changes by at most 0.00001 of it.  *nsweep receives the reference's
 * nsweep, *resab the last sum |res|.  The recurrences run as wavefronts
 * (hyperplanes x+y+z = const), one CTA per block.  Constant coefficients
 * only (H3D_ERR_BAD_CONFIG for L_LSM handles). */
int h3d_mg_sipsol(h3d_mg* h, int32_t nswp, int32_t* nsweep, double* resab);
/* pressure_1sweep (press.for:382-519) on the resident fields, without the
 * boundu/v/w that follow it: pp = 0, calvel, then at most niter times
 * calmas (stop when rmax < eps after the first), sipsol(44), p = p + pp over
 * the block and its ghost layer, pp = 0, exchange(4) + pbound, calvel.
 * info->outer = iterations, info->cycles = SIP sweeps in all, info->rmax the
 * last calmas's, info->relres = ||su||2 of the last calmas; the rmax history
 * is read with h3d_mg_history.  rmax above 10 gives H3D_ERR_DIVERGED. */
int h3d_mg_pressure_1sweep(h3d_mg* h, double dt, double alfapr, double eps, int32_t niter, int32_t nswp,
                           h3d_solve_info* info);

/* --- reference subroutines on the resident level state ----------------- */
/* Canonical level arrays of block ib at level g; field 0 = phi, 1 = rhs. */
int h3d_mg_put_level(h3d_mg* h, int32_t g, int32_t field, int32_t ib, const double* a);
int h3d_mg_get_level(h3d_mg* h, int32_t g, int32_t field, int32_t ib, double* a);
int h3d_mg_mgrelax(h3d_mg* h, int32_t g, int32_t it);   /* mgsolver.for:374-621 */
int h3d_mg_mgrestr(h3d_mg* h, int32_t g);               /* mgsolver.for:623-766 */
int h3d_mg_mgcorr(h3d_mg* h, int32_t g);                /* mgsolver.for:768-910 */
int h3d_mg_mgbound(h3d_mg* h, int32_t g);               /* mgsolver.for:912-997 */
int h3d_mg_exchangepp(h3d_mg* h, int32_t g);            /* exchangepp.for:2-2835 */
int h3d_mg_vcycle(h3d_mg* h);                           /* mgkcyc body on level state */
int h3d_mg_sync(h3d_mg* h);

/* --- failure detection --------------------------------------------------- */
/* Limit, in SM clocks, of every bounded device wait (the mbarrier waits of the
 * TMA-staged kernels) on this handle's GPU; <= 0 restores the default 2^26
 * (tens of milliseconds, where a plane copy takes microseconds).  A wait that
 * runs out makes the call return H3D_ERR_TIMEOUT; the kernel finishes (after
 * the copies it issued have landed) and the handle stays usable.  The limit
 * lives in the library's device memory: it applies to every handle on that
 * GPU.  No counterpart in the reference (its waits are MPI_WAIT). */
int h3d_mg_set_wait_limit(h3d_mg* h, int64_t clocks);
/* Runs one bounded wait that cannot complete (an mbarrier nothing arrives
 * at) with the current limit: returns H3D_ERR_TIMEOUT once the limit has run
 * out, the way a sweep whose plane copy never lands would, and the handle
 * stays usable.  For checking the failure path; no counterpart in the
 * reference. */
int h3d_mg_wait_probe(h3d_mg* h);

/* --- profiling ----------------------------------------------------------- */
/* 1: bracket every full level-1 sweep (not the first one from a zero
 * iterate) with CUDA events on the solve stream and add its duration to
 * h3d_solve_info.smoother_ms. */
int h3d_mg_set_profiling(h3d_mg* h, int32_t on);
/* Smoother kernel variant and z-chunk of level g (the autotuner's choice is
 * the default; H3D_ERR_ARG if the variant cannot run this level).  *nvariants
 * receives the number of variants. */
int h3d_mg_set_smoother(h3d_mg* h, int32_t g, int32_t variant, int32_t zchunk);
int h3d_mg_get_smoother(h3d_mg* h, int32_t g, int32_t* variant, int32_t* zchunk, int32_t* nvariants);
/* Restriction kernel variant and coarse z-chunk used into level g (g >= 2);
 * chosen by timing on large levels in h3d_mg_coeff.  H3D_ERR_ARG if the
 * variant cannot run there.  Tuning controls; no counterpart in the reference. */
int h3d_mg_set_restriction(h3d_mg* h, int32_t g, int32_t variant, int32_t zchunk);
int h3d_mg_get_restriction(h3d_mg* h, int32_t g, int32_t* variant, int32_t* zchunk, int32_t* nvariants);
/* Algorithmic bytes of one level-1 smoother launch (sum over blocks). */
int h3d_mg_smoother_bytes(h3d_mg* h, double* bytes_per_launch);

/* --- host-only helpers (no GPU needed) ---------------------------------- */
/* read_infodom neighbour discovery (alloc_dom.for:524-1200) on integer block
 * extents ext[6*ib..] = xs,xe,ys,ye,zs,ze (global cell units), global bc[6]. */
int h3d_topology(int32_t nblocks, const int32_t* ext, const int32_t* bc,
                 const double* h, int32_t ngrid, h3d_block_desc* out);
/* Ghost-fill gather table of level g, in the canonical packed numbering
 * (blocks concatenated, each (nz+2)(ny+2)(nx+2) x fastest).
 * kind 0: mgbound followed by exchangepp (after every sweep, mgsolver.for:614-615)
 * kind 1: exchangepp alone;  kind 2: mgbound alone;  kind 3: face ghosts of
 * kind 0 (the pressure halo of the outer residual).
 * Entry e: dst[e] <- src[e]; bit 31 of src set = the pre-fill value of that
 * (ghost) cell, clear = the cell's current (interior) value.
 * With dst == NULL only *n is returned. */
int h3d_halo_table(int32_t nblocks, const h3d_block_desc* blocks, int32_t g,
                   int32_t kind, uint32_t* dst, uint32_t* src, int64_t cap,
                   int64_t* n);
/* Expression form of the same fill (kinds 0, 1, 2), which levels with local
 * mesh refinement use: exchangepp between blocks of different rdv averages,
 * injects, extrapolates and interpolates (exchangepp.for:164-189, 447-458,
 * 2115-2123).  A reference r is, by bits 31..30: 00 the current value of cell
 * r, 10 the pre-fill value of cell r & 0x3fffffff, 01 node r & 0x3fffffff,
 * 11 zero (a receive-buffer entry this exchange never wrote).  Node k is
 * nodes[9k..9k+8] = op, operands: 0 copy a0; 1 (a0+...+a7)*0.125; 2 2*a0;
 * 3 ((a0 + 3*a1) - a2)/4; 4 (27a0+9a1+9a2+3a3+9a4+3a5+3a6+1a7)/64, sums left
 * to right.  Nodes only read nodes of lower index.  Write e: dst[e] <- src[e]
 * (a current cell, a node or zero).  nodes == NULL or dst == NULL skips that
 * output; *nnodes and *n are always returned. */
int h3d_halo_expr(int32_t nblocks, const h3d_block_desc* blocks, int32_t g,
                  int32_t kind, uint32_t* nodes, int64_t node_cap, int64_t* nnodes,
                  uint32_t* dst, uint32_t* src, int64_t cap, int64_t* n);

/* Residual norms of one block without allocating device memory.  For hosts
 * that cannot call cudaMalloc: code running under a memory pool whose budget
 * was committed at start-up, or an embedding that forbids device allocation
 * after initialisation.  No counterpart in the reference.
 *   p: device array (nz+2, ny+2, nx+2), x fastest, one ghost layer; b: device
 *   array of the same shape (interior read); h = dx, dy, dz; phys_mask bit f
 *   (W,E,S,N,B,T) = wall face (zero coefficient); out (host) receives
 *   {sum r^2, sum b^2, max|r|*dx*dy*dz, sum r} of r = b - A p (a NaN in r
 *   shows in every entry); stream may be 0.
 * Its per-row partial sums live in a fixed 2 MiB device array inside this
 * library (held by every GPU that loads it until exit), so ny*nz must not
 * exceed 65536 (H3D_ERR_ARG otherwise).  The first call on a device looks up
 * that array's device address and the device's multiprocessor count.  Calls
 * that overlap on the GPU share the array and race.  The call copies its
 * result into `out` on `stream` and synchronises that stream before it
 * returns, so it cannot run on a stream that is being captured into a CUDA
 * graph: it then returns H3D_ERR_ARG without doing anything. */
int h3d_residual_noalloc(const double* p, const double* b, int32_t nx, int32_t ny, int32_t nz,
                         const double* h, int32_t phys_mask, double* out, void* stream);

const char* h3d_mg_strerror(int code);
/* Text of the last error on this handle (or of the last create failure). */
const char* h3d_mg_last_error(const h3d_mg* h);

#ifdef __cplusplus
}
#endif
#endif
