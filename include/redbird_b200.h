/*
 * redbird_b200.h - C ABI of the B200 (sm_100a) FEM forward / Jacobian /
 * Gauss-Newton engine that stands behind the redbirdpy-compatible Python API
 * in redbirdpy_b200/.
 *
 * Conventions
 *   - Every pointer is a DEVICE pointer unless its comment says "host".
 *   - Indices are 0-based int32 (redbirdpy keeps 1-based indices in its cfg
 *     dict; the host layer subtracts 1 once when it uploads).
 *   - Dense multi-column arrays are row-major with the column index fastest:
 *     X[i * ld + c] for node i, column c.  This is numpy's C order of
 *     redbirdpy's Nn x Ncol `phi` and `rhs` arrays.
 *   - Complex values are interleaved (re, im) pairs of the same type
 *     (numpy complex128 / complex64 layout).
 *   - `stream` is a cudaStream_t passed as void*; every call is asynchronous
 *     on that stream unless noted.  No entry point allocates device memory
 *     except where its comment says so; scratch comes from a caller-owned
 *     workspace sized by the matching *_work_bytes() query.
 *   - Return value: RB_OK or one of the RB_E* codes below; rb_last_error()
 *     gives a human-readable message for the calling thread.
 */
#ifndef REDBIRD_B200_H
#define REDBIRD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum rb_status {
  RB_OK = 0,
  RB_EARG = 1,       /* invalid argument (the message names it) */
  RB_ECUDA = 2,      /* a CUDA runtime call failed */
  RB_ESIZE = 3,      /* a size limit of this implementation was exceeded */
  RB_ENOCONV = 4,    /* iterative solve hit its iteration cap (femsolve flag 1) */
  RB_EBREAKDOWN = 5, /* Krylov breakdown (zero or non-finite pivot) */
  RB_ENOTSPD = 6     /* Cholesky met a non-positive pivot */
};

enum rb_scalar { RB_F64 = 0, RB_C128 = 1, RB_F32 = 2, RB_C64 = 3 };
enum rb_propkind { RB_PROP_NODE = 0, RB_PROP_ELEM = 1 };
enum rb_precision { RB_MIXED = 0, RB_FP64 = 1 };

const char* rb_last_error(void);
int rb_version(void);

/* ------------------------------------------------------------------ mesh
 * Tetrahedral mesh resident on the device.  The incidence lists and the CSR
 * pattern are produced once by rb_incidence / rb_csr_pattern_* and reused by
 * every assembly.
 */
typedef struct rb_mesh {
  int64_t nn, ne, nf, nnz;
  const double* node;        /* nn x 3 (mm) */
  const int32_t* elem;       /* ne x 4 */
  const int32_t* face;       /* nf x 3 boundary triangles */
  const double* area;        /* nf */
  const int32_t* node_eptr;  /* nn+1: node -> incident tets */
  const int32_t* node_elist; /* 4*ne, each node's tets ascending */
  const int32_t* node_fptr;  /* nn+1: node -> incident boundary faces */
  const int32_t* node_flist; /* 3*nf, ascending */
  const int32_t* indptr;     /* nn+1 CSR row pointer */
  const int32_t* indices;    /* nnz CSR column indices, ascending per row */
  /* Optional assembly tables from rb_assembly_tables (NULL: not used):
   * inc_slot[node_eptr[n] + u] packs, one byte each, the CSR slots within
   * row n of the 4 nodes of n's u-th incident tet; slot_mask[p] has bit u
   * set when that tet holds column indices[p]. */
  const uint32_t* inc_slot;  /* 4*ne */
  const uint32_t* slot_mask; /* nnz */
} rb_mesh;

/* Node -> cell incidence (cells are tets, nv=4, or triangles, nv=3):
 * ptr[n]..ptr[n+1] lists the cells that contain node n, ascending.
 * Replaces the per-element Python loop of `_femnz` (redbirdpy/utility.py:1020-1041)
 * as the structure the assembly walks. */
size_t rb_incidence_work_bytes(int64_t ncell, int32_t nv, int64_t nn);
int rb_incidence(const int32_t* cells, int32_t nv, int64_t ncell, int64_t nn,
                 int32_t* ptr, int32_t* list, void* work, size_t work_bytes, void* stream);

/* CSR sparsity of the FEM matrix: row n holds every node that shares a tet
 * with n (diagonal included), columns ascending.  Bit-identical to the
 * indptr/indices scipy produces for femlhs's COO -> tocsr
 * (redbirdpy/forward.py:254).  count fills indptr[0..nn]; the host reads
 * indptr[nn] (= nnz), allocates indices and calls fill. */
size_t rb_csr_pattern_work_bytes(int64_t nn);
int rb_csr_pattern_count(const int32_t* elem, int64_t nn, const int32_t* node_eptr,
                         const int32_t* node_elist, int32_t* indptr, void* work,
                         size_t work_bytes, void* stream);
int rb_csr_pattern_fill(const int32_t* elem, int64_t nn, const int32_t* node_eptr,
                        const int32_t* node_elist, const int32_t* indptr, int32_t* indices,
                        void* stream);

/* ------------------------------------------------------------- assembly */
/* Incidence tables that let femlhs sum each matrix entry over only the tets
 * that hold it.  Fills inc_slot (4*ne) and slot_mask (nnz) and sets *usable
 * to 1 when every node has at most 32 incident tets and every row at most
 * 255 columns (the tables' limits); with *usable 0 the mesh is assembled
 * without them (leave rb_mesh.inc_slot / slot_mask NULL).  Synchronises
 * the stream. */
int rb_assembly_tables(const rb_mesh* mesh, uint32_t* inc_slot, uint32_t* slot_mask, int32_t* usable,
                       void* stream);

typedef struct rb_optics {
  int32_t kind;        /* RB_PROP_NODE: arrays have nn entries; RB_PROP_ELEM: ne */
  const double* mua;   /* 1/mm */
  const double* musp;  /* reduced scattering mus*(1-g), 1/mm */
  const double* nref;  /* per node/elem refractive index, or NULL */
  double nref_scalar;  /* used when nref == NULL */
  double omega;        /* modulation angular frequency (rad/s); > 0 -> complex */
  double reff;         /* effective reflection coefficient of the boundary */
} rb_optics;

/* Per-tet mua and musp from a label table (the label branch of femlhs,
 * redbirdpy/forward.py:127-140: prop[seg]): mua_out[e] = tab[l][0],
 * musp_out[e] = tab[l][1] * (1 - tab[l][2]) with l = seg[e] clipped to
 * [0, nlabel).  tab is nlabel x ncol (ncol >= 2; g is taken as 0 when
 * ncol == 2), all on the device. */
int rb_prop_from_labels(const int32_t* seg, int64_t ne, const double* tab, int64_t nlabel, int32_t ncol,
                        double* mua_out, double* musp_out, void* stream);

/* femlhs (redbirdpy/forward.py:90-256): A = K*D + M*mua (+ i*omega/c*n*M)
 * + Robin boundary terms, written into the fixed CSR pattern of `mesh`.
 * Like the reference it combines the precomputed deldotdel rows `ddd`
 * (ne x 10) and tet volumes `evol` (ne) with the current properties.  One
 * warp per matrix row gathers the contributions of the row's tets and
 * boundary faces in a fixed order, so results are deterministic.
 *   val64  nnz doubles (real) or nnz complex128 (omega > 0), required
 *   val32  optional FP32 / complex64 copy for the mixed-precision solver
 *   dinv64 optional nn reciprocal diagonal (Jacobi), same scalar kind
 *   dinv32 optional FP32 copy of dinv64
 *   work   rb_femlhs_work_bytes(nn, ne) bytes of scratch */
size_t rb_femlhs_work_bytes(int64_t nn, int64_t ne);
int rb_femlhs(const rb_mesh* mesh, const rb_optics* optics, const double* evol, const double* ddd,
              void* val64, void* val32, void* dinv64, void* dinv32, void* work, size_t work_bytes,
              void* stream);

/* rb_femlhs without a workspace, for callers that cannot allocate device
 * memory (no counterpart in the reference): the scratch array comes from a
 * fixed 32 MiB device array inside this library, enough for 4,194,304 nodes
 * (per-node properties) or tets (per-tet properties); larger meshes get
 * RB_ESIZE.  The first call on each device looks up that array's address and
 * should therefore come before any stream capture.  All calls share the one
 * array, so calls that overlap on the GPU (different streams or threads
 * without ordering between them) race; calls on one stream are safe.
 * Allocates nothing (no cudaMalloc/cudaFree). */
int rb_femlhs_noalloc(const rb_mesh* mesh, const rb_optics* optics, const double* evol,
                      const double* ddd, void* val64, void* val32, void* dinv64, void* dinv32,
                      void* stream);

/* meshprep on the device (redbirdpy/utility.py:101-246 with the reference's
 * fallbacks, utility.py:1005-1109), all index arrays 0-based int32:
 *   rb_reorient    swap nodes 0 and 1 of tets of negative signed volume, in
 *                  place (elem ne x 4, 16-byte aligned); evol (optional)
 *                  receives |V|; flipped (optional, device) counts the swaps
 *   rb_volface     boundary triangles (each tet's faces (0,2,1), (0,1,3),
 *                  (0,3,2), (1,2,3); those whose sorted node triple occurs
 *                  once), in the order of their sorted triples, each with its
 *                  tet's orientation; face holds 4 ne x 3 int32, *nf (host)
 *                  the count; nn < 2^21
 *   rb_face_area   triangle areas
 *   rb_nodevolume  nvol[n] = 1/4 sum of evol over the tets of node n
 *                  (incidence lists of rb_incidence)
 * The arithmetic follows numpy's order without fused multiply-adds: the
 * results carry the bits of the host fallbacks. */
int rb_reorient(const double* node, int32_t* elem, int64_t ne, double* evol, int32_t* flipped, void* stream);
size_t rb_volface_work_bytes(int64_t ne);
int rb_volface(const int32_t* elem, int64_t ne, int64_t nn, int32_t* face, int64_t* nf /* host */, void* work,
               size_t work_bytes, void* stream);
int rb_face_area(const double* node, const int32_t* face, int64_t nf, double* area, void* stream);
int rb_nodevolume(int64_t nn, const int32_t* node_eptr, const int32_t* node_elist, const double* evol,
                  double* nvol, void* stream);

/* deldotdel (redbirdpy/utility.py:53-98): ne x 10 values V*grad(phi_i).grad(phi_j)
 * for the pairs (0,0),(0,1),(0,2),(0,3),(1,1),(1,2),(1,3),(2,2),(2,3),(3,3),
 * from the node coordinates; evol (optional, ne) receives |V| like
 * elemvolume (utility.py:1090-1109). */
int rb_deldotdel(const double* node, const int32_t* elem, int64_t ne, double* ddd, double* evol,
                 void* stream);

/* ------------------------------------------------------------ optodes */
/* Point location used by femrhs (iso2mesh.tsearchn at redbirdpy/forward.py:316,337):
 * loc[k] = lowest tet index whose barycentric coordinates of pts[k] are all
 * >= -1e-9 (or -1 when none), bary[k] = those 4 coordinates (NaN when
 * outside).  pts is npts x 3. */
int rb_tsearch(const double* node, const int32_t* elem, int64_t ne, const double* pts,
               int64_t npts, int32_t* loc, double* bary, void* stream);

/* Dense point-optode RHS (femrhs column fill, redbirdpy/forward.py:314-348):
 * B (nn x ld, real, must be zeroed by the caller) gets bary[k][m] at row
 * elem[loc[k]][m], column col0 + k; optodes with loc < 0 leave a zero column. */
int rb_point_rhs(const int32_t* elem, const int32_t* loc, const double* bary, int64_t npts,
                 int64_t nn, int64_t ld, int64_t col0, double* B, void* stream);

/* Wide-field (pattern) sources and detectors: the dense columns of
 * cfg['widesrc'] / cfg['widedet'] (W: nn x w, row stride ldw; femrhs,
 * redbirdpy/forward.py:326-352, where they follow the point columns of their
 * kind).  rb_wide_rhs copies them into B (nn x ld) at column col0;
 * rb_wide_getdet forms their detector rows (femgetdet, forward.py:430-442):
 * detval[d * nsrc + s] = sum_n W[n][d] phi[n * ld + s] for d < wd, phi and
 * detval of scalar kind `kind` (RB_F64 or RB_C128), deterministic. */
int rb_wide_rhs(const double* W, int64_t nn, int64_t w, int64_t ldw, int64_t ld, int64_t col0, double* B,
                void* stream);
size_t rb_wide_getdet_work_bytes(int64_t wd, int64_t nsrc, int32_t kind);
int rb_wide_getdet(const double* W, int64_t nn, int64_t wd, int64_t ldw, const void* phi, int64_t ld,
                   int64_t nsrc, int32_t kind, void* detval, void* work, size_t work_bytes, void* stream);

/* femgetdet (redbirdpy/forward.py:365-442) for point detectors:
 * detval[d * nsrc + s] = sum_m bary_det[d][m] * phi[elem[loc_det[d]][m] * ld + s]
 * phi/detval scalar kind `kind` (RB_F64 or RB_C128). */
int rb_femgetdet(const int32_t* elem, const int32_t* loc_det, const double* bary_det,
                 int64_t ndet, const void* phi, int64_t ld, int64_t nsrc, int32_t kind,
                 void* detval, void* stream);

/* --------------------------------------------------------------- solve */
typedef struct rb_csr {
  int64_t n, nnz;
  const int32_t* indptr;
  const int32_t* indices;
  const void* val64;   /* FP64 / complex128 values */
  const void* val32;   /* FP32 / complex64 copy (required for RB_MIXED) */
  const void* dinv64;  /* reciprocal diagonal, FP64 kind */
  const void* dinv32;  /* reciprocal diagonal, FP32 kind (required for RB_MIXED) */
  int32_t is_complex;
} rb_csr;

/* Coarse space of the two-level preconditioner: the rows are grouped into nc
 * aggregates (e.g. the mesh nodes binned by position).  With P the n x nc 0/1
 * matrix of the grouping, the Krylov preconditioner becomes
 *   z = D^-1 r + P (P^T A P)^-1 P^T r
 * (Jacobi plus an exact solve of the aggregated operator, which removes the
 * smooth error components Jacobi-CG converges on slowly).  P^T A P is built
 * and inverted on the device once per rb_femsolve call.  Device arrays. */
typedef struct rb_coarse {
  int64_t nc;              /* aggregates, 1..4096; every aggregate nonempty */
  const int32_t* agg;      /* n: aggregate of each row (0-based) */
  const int32_t* agg_ptr;  /* nc + 1: offsets into agg_rows */
  const int32_t* agg_rows; /* n: the rows of each aggregate, ascending */
} rb_coarse;

/* Workspace that a coarse space adds to rb_femsolve_work_bytes(). */
size_t rb_coarse_work_bytes(int64_t nc, int64_t nrhs, int32_t is_complex, int32_t precision);

/* Aggregates from node positions (node: nn x 3 FP64, device): node i falls
 * in the cube (bx, by, bz) = floor((p - (x0, y0, z0)) / h), clamped to the
 * nbx x nby x nbz grid; the nonempty cubes, numbered in cube order
 * (x fastest), are the aggregates.  Writes agg (nn), agg_ptr (nc + 1; room
 * for 4097) and agg_rows (nn, each aggregate's rows ascending), and *nc
 * (host).  Deterministic.  RB_ESIZE when more than 4096 cubes are nonempty
 * (*nc holds the count: take a larger h). */
size_t rb_coarse_aggregate_work_bytes(int64_t nn, int64_t nbins);
int rb_coarse_aggregate(const double* node, int64_t nn, double x0, double y0, double z0, double h,
                        int32_t nbx, int32_t nby, int32_t nbz, int32_t* agg, int32_t* agg_ptr,
                        int32_t* agg_rows, int64_t* nc /* host */, void* work, size_t work_bytes,
                        void* stream);

/* Spatial row groups of the blocked SpMM inside rb_femsolve (no counterpart
 * in the reference, whose solves run in SuperLU): up to 8 rows per group, the
 * nodes of one cube of edge about two node spacings, so that one warp gathers
 * each x row of the group's column union once for all its rows.  Built once
 * per mesh (rb_rowgroups_bin) and per CSR pattern (rb_rowgroups_union_*).
 * Device arrays; coef is scratch that every rb_femsolve call using the groups
 * overwrites (nu x 8 values of the solve's FP32 kind: 32 bytes per entry for
 * real, 64 for complex), so solves sharing one rb_rowgroups must not overlap
 * on the GPU. */
typedef struct rb_rowgroups {
  int64_t ng;             /* groups */
  const int32_t* rows;    /* ng x 8 row indices, -1 pads a short group */
  const int32_t* uptr;    /* ng + 1: each group's union entries */
  const int32_t* ucol;    /* nu columns, ascending within a group */
  const uint8_t* umask;   /* nu: bit r set when row r of the group holds the column */
  int64_t nu;             /* union entries (uptr[ng]) */
  void* coef;             /* nu x 8 scratch (see above) */
} rb_rowgroups;

/* Groups from node positions (node: nn x 3 FP64, device): node i falls in the
 * cube floor((p - (x0, y0, z0)) / h), clamped to the nbx x nby x nbz grid;
 * each cube's nodes, ascending, are cut into groups of 8 (the last one short).
 * Groups follow the cubes in blocks of 2 x 2 x 2 cubes (x fastest inside a
 * block and between blocks).  rows must hold 8 nn int32; *ng (host) receives
 * the group count.  nbins = nbx nby nbz for the workspace query.
 * Deterministic. */
size_t rb_rowgroups_work_bytes(int64_t nn, int64_t nbins);
int rb_rowgroups_bin(const double* node, int64_t nn, double x0, double y0, double z0, double h,
                     int32_t nbx, int32_t nby, int32_t nbz, int32_t* rows, int64_t* ng /* host */,
                     void* work, size_t work_bytes, void* stream);
/* Column unions of the groups over A's pattern: count writes uptr (ng + 1)
 * and *nu (host); fill writes ucol and umask (nu each). */
size_t rb_rowgroups_union_work_bytes(int64_t ng);
int rb_rowgroups_union_count(const rb_csr* A, const int32_t* rows, int64_t ng, int32_t* uptr,
                             int64_t* nu /* host */, void* work, size_t work_bytes, void* stream);
int rb_rowgroups_union_fill(const rb_csr* A, const int32_t* rows, int64_t ng, const int32_t* uptr,
                            int32_t* ucol, uint8_t* umask, void* stream);
/* Independent systems stacked block-diagonally in one matrix (a batch of
 * instances): rows row_ptr[i] .. row_ptr[i+1]-1 belong to instance i.  With
 * it the refinement tests ||b_i - A_i x_i|| / ||b_i|| of every (instance,
 * column) on its own, scales each instance's correction right-hand side to
 * unit norm on its rows, and stops correcting an instance's column once it
 * is done, so that an instance's accuracy does not depend on the others.
 * The caller adds rb_instances_work_bytes to the femsolve workspace. */
typedef struct rb_instances {
  int64_t ninst;
  const int64_t* row_ptr;  /* device, ninst+1, ascending, row_ptr[ninst] = n */
  const int32_t* row_inst; /* device, n: the instance of each row */
  int32_t* status;         /* device out, ninst: 0 converged, 1 not converged within
                              the sweep / iteration caps, 2 Krylov breakdown,
                              3 non-finite residual, 4 a bounded in-kernel wait
                              gave up (results invalid) */
  double* relres;          /* device out, ninst x nrhs (row-major), or NULL: the final
                              ||b_i - A_i x_i|| / ||b_i|| per (instance, column) */
} rb_instances;
size_t rb_instances_work_bytes(int64_t ninst, int64_t nrhs);

typedef struct rb_solve_opts {
  int32_t precision;   /* RB_MIXED: FP32 Krylov + FP64 refinement; RB_FP64 */
  int32_t max_outer;   /* refinement sweeps (mixed) */
  int32_t maxiter;     /* cap on Krylov iterations per sweep */
  int32_t check_every; /* iterations between host convergence checks; 0: a fixed
                          budget of max_outer sweeps x maxiter iterations with no
                          host check or read-back at all (the call only queues
                          work: it can be captured into a CUDA graph); converged
                          columns turn the remaining launches into no-ops.  Needs
                          instances (the outcome is in their status words) and
                          no coarse space; info->flag and relres are -1. */
  double tol;          /* target max relative residual ||b-Ax||/||b|| */
  double inner_tol;    /* relative residual of each FP32 correction solve */
  int32_t profile;     /* nonzero: time the Krylov kernels with CUDA events */
  int32_t use_x0;      /* nonzero: X holds an initial guess (e.g. the previous
                          Gauss-Newton iterate's fields); zero: start from 0 */
  const rb_coarse* coarse; /* host pointer; NULL: Jacobi preconditioner only */
  const rb_rowgroups* groups; /* host pointer; NULL: the SpMM walks rows (or row pairs) */
  const rb_instances* instances; /* host pointer; NULL: one system */
  int32_t spmm_lanes;  /* lanes per row of the per-row SpMM (4, 8, 16 or 32; each
                          takes ceil(nrhs / lanes) columns, 1, 2 or 4 of them);
                          0: chosen from nrhs.  Row-pair and row-group
                          products ignore it. */
} rb_solve_opts;

typedef struct rb_solve_info {
  int32_t iters;       /* total Krylov iterations */
  int32_t outer;       /* refinement sweeps done */
  int32_t flag;        /* femsolve flag: 0 converged, 1 iteration cap, 2 breakdown */
  int32_t launches;    /* kernels launched by this call */
  double relres;       /* max over columns of ||b-Ax||/||b|| (FP64) */
  double spmm_ms;      /* profile only: total time of the SpMM launches */
  double update_ms;    /* profile only: total time of the vector-update launches */
  int32_t spmm_launches;
  int32_t update_launches;
  double coarse_ms;    /* profile only: total time of the coarse corrections */
  int32_t coarse_launches; /* profile only: coarse corrections timed */
  int32_t sweep_iters_max; /* the most Krylov iterations one refinement sweep took */
} rb_solve_info;

/* femsolve (redbirdpy/solver.py:385-948) for all columns at once: Jacobi-
 * preconditioned block CG (real SPD) or block COCG (complex symmetric,
 * unconjugated bilinear form).  B is nn x nrhs real FP64; X is nn x nrhs of
 * the matrix's FP64 kind.  All-zero columns of B give exactly zero columns
 * (the reference skips them, solver.py:568-581). */
size_t rb_femsolve_work_bytes(int64_t n, int64_t nnz, int64_t nrhs, int32_t is_complex, int32_t precision);
int rb_femsolve(const rb_csr* A, const double* B, void* X, int64_t nrhs,
                const rb_solve_opts* opts, rb_solve_info* info /* host */, void* work,
                size_t work_bytes, void* stream);

/* FP32 (complex64) copy of the values and the reciprocal diagonal of a CSR
 * matrix given in FP64 (for matrices that did not come from rb_femlhs).
 * Any of val32 / dinv64 / dinv32 may be NULL. */
int rb_csr_prepare(const rb_csr* A, void* val32, void* dinv64, void* dinv32, void* stream);

/* Y = A X for nrhs columns (rows of X/Y contiguous, ld = nrhs).
 * kind: RB_F64/RB_C128 use val64, RB_F32/RB_C64 use val32. */
int rb_spmm(const rb_csr* A, int32_t kind, const void* X, void* Y, int64_t nrhs, void* stream);

/* ------------------------------------------------------------ Jacobian */
/* Adjoint Jacobian rows (jac, redbirdpy/forward.py:509-569) written straight
 * to nodes, without the nsd x ne element matrix:
 *   what RB_JAC_MUA_REF:   the reference's mua Jacobian,
 *       Jn[k][n] = 1/4 sum_{tets e of n} Je[k][e],
 *       Je[k][e] = -0.1 V_e (sum_i ps_i pd_i + 1/2 sum_{i!=j} ps_i pd_j)
 *   what RB_JAC_MUA_NODAL: exact derivative of the node-based femlhs assembly
 *       (forward.py:177-228 lumped mass weights) with respect to nodal mua at
 *       fixed D
 *   what RB_JAC_D:         exact derivative with respect to nodal diffusion
 *       coefficient D: JD[k][n] = -1/4 sum_{tets e of n} ps_e^T K_e pd_e,
 *       K_e = V grad(l_i).grad(l_j)
 * Column map: the pairs read nc phi columns cols[0..nc); the ndet detector
 * columns are the slots det0..det0+ndet-1.  Pair k uses source slot
 * pair_src[k] (0..nc-1) and detector pair_det[k] (0..ndet-1).  J is nsd rows
 * of leading dimension ldj >= nn (row k at J + k*ldj).  Passing nsd as the
 * negative of nsrc*ndet declares that the pairs are every (source slot,
 * detector) combination in detector-major order, k = d*nsrc + s, with nsrc
 * = det0 and both counts multiples of 4 (sdmap's layout); this selects a
 * register-blocked path.  rmax / emax: the
 * largest CSR row length and the largest number of tets at one node.
 * phi_kind / out_kind: any real kind with a real kind, complex with complex;
 * out RB_F32/RB_C64 computes in FP32.  evol: ne tet volumes; ddd: the ne x 10
 * deldotdel rows (required for RB_JAC_D only), as jac receives them. */
enum rb_jac_what { RB_JAC_MUA_REF = 0, RB_JAC_MUA_NODAL = 1, RB_JAC_D = 2 };
/* extra out_kind values for complex phi: real FP32 / FP64 output with the
 * real parts in rows 0..nsd-1 and the imaginary parts in rows nsd..2nsd-1
 * (matreform 'real' stacking, redbirdpy/recon.py:532-546) */
enum rb_jac_split { RB_JAC_SPLIT_F32 = 4, RB_JAC_SPLIT_F64 = 5,
                    RB_JAC_SPLIT_BF16 = 6, /* split rows rounded to BF16 (GN step in BF16) */
                    RB_JAC_BF16 = 7, /* real rows rounded to BF16 */
                    RB_JAC_SPLIT_F32_ACC64 = 8, /* split FP32 rows whose products are formed
                                                   in FP64 (only the storage rounds) */
                    RB_JAC_F32_ACC64 = 9 /* real FP32 rows, products formed in FP64 */ };
int rb_jac(const rb_mesh* mesh, int32_t what, const void* phi, int32_t phi_kind, int64_t ld,
           const int32_t* cols, int32_t nc, int32_t det0, int32_t ndet, const int32_t* pair_src,
           const int32_t* pair_det, int64_t nsd, void* J, int64_t ldj, int32_t out_kind,
           int32_t rmax, int32_t emax, const double* evol, const double* ddd, void* stream);
/* Pair products on the tensor cores: rb_jac / rb_jac_range take them
 * (tcgen05 kind::tf32 with a hi/lo split of both operands, FP32 accuracy)
 * when the pairs are the full source x detector grid (nsd < 0), the output
 * is FP32 (RB_F32, or RB_JAC_SPLIT_F32 for complex fields), there are at
 * most 128 sources and 64 detectors (128 for real fields) and rmax <= 32;
 * otherwise the SIMT products.  rb_jac_tensor_cores(1) allows the tensor
 * cores, 0 (the default) keeps the SIMT products.  The tensor-core
 * kernel's waits are bounded: rb_jac_status synchronises the stream and
 * returns RB_ECUDA (and clears the word) if one gave up since the last call. */
int rb_jac_tensor_cores(int32_t on);
int rb_jac_status(void* stream);
/* rb_jac for the nodes node0 .. node0+count-1 only: J column c holds node
 * node0 + c (ldj >= count).  A GN step whose full J would not fit in HBM
 * forms its products from node slabs recomputed on demand. */
int rb_jac_range(const rb_mesh* mesh, int32_t what, const void* phi, int32_t phi_kind, int64_t ld,
                 const int32_t* cols, int32_t nc, int32_t det0, int32_t ndet, const int32_t* pair_src,
                 const int32_t* pair_det, int64_t nsd, void* J, int64_t ldj, int32_t out_kind,
                 int32_t rmax, int32_t emax, const double* evol, const double* ddd, int64_t node0,
                 int64_t count, void* stream);

/* Dual-mesh Jacobian remap (_remap_jacobian, redbirdpy/recon.py:818-876):
 * out[r][q] = sum_{p in [map_ptr[q], map_ptr[q+1])} map_w[p] J[r][map_idx[p]]
 * for rows r < rows and reconstruction nodes q < nq; map_idx lists the
 * forward nodes whose enclosing reconstruction element has node q (map_w:
 * that node's barycentric weight), ascending.  J and out of kind `kind`
 * (RB_F32, RB_C64, RB_F64 or RB_C128), row strides ldj and ldo. */
int rb_jac_remap(const void* J, int32_t kind, int64_t rows, int64_t ldj, const int32_t* map_ptr,
                 const int32_t* map_idx, const double* map_w, int64_t nq, void* out, int64_t ldo,
                 void* stream);
/* One wavelength's Jacobian rows into the stacked real GN matrix (FP32 rows,
 * ldd): with v = src[r][c] (scale_re + i scale_im) rowscale[r] (rowscale:
 * optional complex per-row factors, re/im pairs), dst[row_re + r][col0 + c]
 * = Re v and, when row_im >= 0, dst[row_im + r][col0 + c] = Im v.  Covers
 * jacchrome's extinction weights (redbirdpy/forward.py:572-589) and
 * matreform's forms (recon.py:512-567): 'real' stacking, 'reim' (second
 * column block with the factor i), 'logphase' (rowscale conj(y)/|y|^2).
 * src RB_F32 or RB_C64, row stride lds. */
int rb_jac_block(const void* src, int32_t kind, int64_t rows, int64_t cols, int64_t lds, double scale_re,
                 double scale_im, const double* rowscale, float* dst, int64_t ldd, int64_t row_re,
                 int64_t row_im, int64_t col0, void* stream);

/* Element Jacobian Je (nsd x ne, kind of phi: RB_F64 or RB_C128), the second
 * output of jac (forward.py:527-557); src_col/det_col are phi columns. */
int rb_jac_elem(const rb_mesh* mesh, const double* evol, const void* phi, int32_t phi_kind, int64_t ld,
                const int32_t* src_col, const int32_t* det_col, int64_t nsd, void* je,
                void* stream);

/* Adjoint fields of the backward pass (no counterpart in the reference, which
 * has no autograd): for the instance i that owns row r (rows
 * [row0[i], row0[i+1]), detector rows [det0[i], det0[i+1]) of g),
 *   lam[r][s] = sum_d phi[r][dcol0 + d] * conj(g[det0[i] + d][s]),  s < ns
 * i.e. lambda_s = A^-1 sum_d conj(g[d, s]) b_d from the detector columns of
 * the forward solve.  phi: nn x ld, g: ndet_total x ns, lam: nn x ns, all
 * RB_F64 or all RB_C128 (kind).  ninst = 1 for a single mesh. */
int rb_adjoint_fields(const void* phi, int64_t nn, int64_t ld, int64_t dcol0, const void* g, int64_t ns,
                      const int64_t* row0, const int64_t* det0, int64_t ninst, int32_t kind, void* lam,
                      void* stream);

/* ------------------------------------------------------ Gauss-Newton step
 * reginvunder (redbirdpy/recon.py:429-509) on the device:
 *   H = alpha J J^T            rb_gram: tcgen05 tensor cores, TF32 inputs,
 *                              FP32 accumulation, FP64 output (all of H).
 *                              With Jlo != NULL (J = hi + lo, from
 *                              rb_split_tf32) H = hi hi^T + hi lo^T + lo hi^T,
 *                              close to FP32-input accuracy at 3x the work.
 *                              J: M x K FP32 rows, ldj % 4 == 0, 16-B aligned.
 *                              rb_gram_bf16: J stored as BF16 (kind::f16 with
 *                              BF16 A and B), ldj % 8 == 0: half the bytes and
 *                              twice the tensor rate of TF32.
 *   H += lambda I, normalise   rb_reginv_prepare (_normalize_diag, recon.py:784-789)
 *   H = L L^T                  rb_cholesky (FP64, in place, lower; the strict
 *                              upper triangle of each 64 x 64 diagonal block
 *                              receives that block's inverse, transposed).  The
 *                              factorization forks onto two library-owned
 *                              streams per device (created on first use: the
 *                              panel steps at the highest priority, the bulk
 *                              trailing updates beside them), joins them back
 *                              into `stream` and synchronizes it before
 *                              returning (it reads the pivot check back)
 *   L L^T x = b                rb_chol_solve (in place on x; L as rb_cholesky
 *                              leaves it, diagonal-block inverses included)
 *   out = alpha J^T y + beta out   rb_gemv_t (J aligned as for rb_gram; ldj % 4 == 0)
 *   sum(J^2)                   rb_sumsq (Frobenius block scale, recon.py:235) */
size_t rb_gram_work_bytes(void);
int rb_gram(const float* J, const float* Jlo, int64_t M, int64_t K, int64_t ldj, double alpha,
            double* H, int64_t ldh, void* work, size_t work_bytes, void* stream);
int rb_gram_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double alpha, double* H, int64_t ldh,
                 void* work, size_t work_bytes, void* stream);
/* Optional staging buffer (same results, bit for bit): the tiles are formed
 * from column slabs of J (65536 wide) copied into a compact buffer first.
 * Long rows (a row stride of megabytes) spread one slab over a page per row;
 * the compact slab halves the time of a slab's products at 8192 x 1,040,502.
 * rb_gram_stage_bytes returns the bytes to pass (0: staging does not pay for
 * this shape; the staged calls then run as the plain ones).  elem_bytes is 4
 * (FP32) or 2 (BF16); split != 0 when Jlo is given. */
size_t rb_gram_stage_bytes(int64_t M, int64_t K, int64_t ldj, int32_t elem_bytes, int32_t split);
int rb_gram_staged(const float* J, const float* Jlo, int64_t M, int64_t K, int64_t ldj, double alpha,
                   double* H, int64_t ldh, void* stage, size_t stage_bytes, void* work, size_t work_bytes,
                   void* stream);
int rb_gram_bf16_staged(const void* J, int64_t M, int64_t K, int64_t ldj, double alpha, double* H,
                        int64_t ldh, void* stage, size_t stage_bytes, void* work, size_t work_bytes,
                        void* stream);
int rb_split_tf32(float* J, float* lo, int64_t M, int64_t K, int64_t ldj, void* stream);
int rb_reginv_prepare(double* H, int64_t M, int64_t ldh, double lambda, double* di, void* stream);
size_t rb_cholesky_work_bytes(void);
int rb_cholesky(double* H, int64_t M, int64_t ldh, void* work, size_t work_bytes, void* stream);
/* rb_chol_solve's workspace: M doubles (the forward solution) */
size_t rb_chol_solve_work_bytes(int64_t M);
int rb_chol_solve(const double* L, int64_t M, int64_t ldh, double* x, void* work, size_t work_bytes, void* stream);
size_t rb_gemv_t_work_bytes(int64_t K);
int rb_gemv_t(const float* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha,
              double beta, double* out, void* work, size_t work_bytes, void* stream);
int rb_gemv_t_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha,
                   double beta, double* out, void* work, size_t work_bytes, void* stream);
size_t rb_sumsq_work_bytes(void);
int rb_sumsq(const float* J, int64_t M, int64_t K, int64_t ldj, double* out, void* work,
             size_t work_bytes, void* stream);
int rb_sumsq_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double* out, void* work,
                  size_t work_bytes, void* stream);
/* rows[m] = sum_k J[m][k]^2 (FP64 accumulation; the exact diagonal of J J^T
 * for the stored rows), and *total = sum_m rows[m] when total != NULL (the
 * Frobenius sum of rb_sumsq, same pass).  A diagonal taken from the
 * tensor-core product carries its input rounding (TF32 ~1e-3 relative), which
 * a regularisation relative to the largest diagonal entry would inherit. */
int rb_row_sumsq(const float* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total, void* stream);
int rb_row_sumsq_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total,
                      void* stream);
/* rb_row_sumsq of FP32 rows that also writes them rounded to BF16 (row
 * stride ldb >= K, a multiple of 8; padding zeroed) in the same pass: the
 * operand of rb_gram_bf16 when the refinement runs over the FP32 rows. */
int rb_row_sumsq_to_bf16(const float* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total, void* bf,
                         int64_t ldb, void* stream);
/* H[i][i] = alpha d[i] */
int rb_set_diag(double* H, int64_t M, int64_t ldh, const double* d, double alpha, void* stream);
int rb_vec_mul(const double* a, const double* b, double* out, int64_t n, void* stream);
/* FP64 iterative refinement of the normal equations (alpha J J^T + lambda I) y = r
 * around the tensor-core factor (the refinement residual r - alpha J (J^T y)
 * - lambda y takes FP64-accumulated products over the stored J, so y reaches
 * the accuracy of J itself; no counterpart in the reference, which solves the
 * FP64 normal matrix directly, recon.py:474-483):
 *   out = alpha J x + beta out     rb_gemv_n (J as for rb_gemv_t, rows padded to
 *                                  a multiple of 4 entries; x FP64, K entries)
 *   y = a x + b y                  rb_axpby
 *   x . y                          rb_dot (the residual norms) */
/* rb_gemv_n's workspace: the per-row parts of each 1024-column chunk
 * (M x ceil(K / 1024) doubles) */
size_t rb_gemv_n_work_bytes(int64_t M, int64_t K);
int rb_gemv_n(const float* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
              double* out, void* work, size_t work_bytes, void* stream);
int rb_gemv_n_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
                   double* out, void* work, size_t work_bytes, void* stream);
int rb_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream);
/* *out = x . y (FP64, device scalar; fixed-order reduction) */
size_t rb_dot_work_bytes(void);
int rb_dot(int64_t n, const double* x, const double* y, double* out, void* work, size_t work_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* REDBIRD_B200_H */
