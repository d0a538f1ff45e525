/*
 * v2rdm_b200 -- C ABI of the B200 boundary-point SDP path for hilbert's
 * v2RDM-CASSCF solver.  Plain pointers and sizes only; every entry point
 * returns a status code (never throws) and v2b_last_error() describes the
 * last failure on the calling thread.
 *
 * Two families of entry points:
 *
 *  1. libsdp-shaped solver (drop-in for libsdp::BPSDPSolver as hilbert calls
 *     it).  The caller supplies A.x / A^T.y as host callbacks exactly like
 *     evaluate_Au / evaluate_ATu (src/v2rdm_casscf/v2rdm_solver.cc:97-112);
 *     vectors stay on the host, the per-block PSD projection runs on the GPU.
 *
 *  2. Device-map problems: the constraint operator of a C1 v2RDM problem is
 *     built in the library (bit-exact to hilbert's maps) and every step of the
 *     iteration -- A.x, A^T.y, conjugate gradients, projection, norms -- runs
 *     on the GPU.  x, b, c passed to v2b_problem_solve are host arrays.
 */
#ifndef V2RDM_B200_H
#define V2RDM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define V2B_OK             0
#define V2B_NOT_CONVERGED  1   /* iteration cap reached (not an error for solve) */
#define V2B_BAD_ARG        2
#define V2B_NAN            3   /* non-finite value met in a reduction */
#define V2B_DEVICE_TIMEOUT 4   /* a bounded device-side wait gave up */
#define V2B_CUDA_ERROR     5
#define V2B_NO_DEVICE      6
#define V2B_INTERNAL       7

/* POSITIVITY option values (src/plugin.cc:220) supported on the device path */
#define V2B_POSITIVITY_D   0
#define V2B_POSITIVITY_DQ  1
#define V2B_POSITIVITY_DG  2
#define V2B_POSITIVITY_DQG 3
#define V2B_POSITIVITY_DQGT2 4   /* DQG + T2 (t2.cc:1236-1843, 3376-3966) */
#define V2B_POSITIVITY_DQGT1 5   /* DQG + T1 (t1.cc:419-795, 795-1200) */
#define V2B_POSITIVITY_DQGT1T2 6 /* DQG + T1 + T2 ("DQGT1T2" and "DQGT", v2rdm_solver.cc:4110-4119) */
/* OR-ed into a POSITIVITY value: CONSTRAIN_D3 (d3.cc:45-406, 408-766) and
 * CONSTRAIN_Q3 (q3.cc:45-423, 425-803; implies D3, needs Q2 and G2) */
#define V2B_CONSTRAIN_D3 16
#define V2B_CONSTRAIN_Q3 32
/* CONSTRAIN_E3 (e3.cc:45-566, 570-1082; implies D3) */
#define V2B_CONSTRAIN_E3 64
/* CONSTRAIN_F3 (f3.cc:45-836, 842-1623; implies D3) */
#define V2B_CONSTRAIN_F3 128
/* CONSTRAIN_D4 (d4.cc:44-297, 300-557; implies D3) */
#define V2B_CONSTRAIN_D4 256

/* libsdp::SDPOptions as hilbert fills it (src/v2rdm_casscf/v2rdm_solver.cc:426-431) */
typedef struct {
    double sdp_objective_convergence; /* E_CONVERGENCE  (src/plugin.cc:94)  */
    double sdp_error_convergence;     /* R_CONVERGENCE  (src/plugin.cc:97)  */
    double cg_convergence;            /* CG_CONVERGENCE (src/plugin.cc:238) */
    int cg_maxiter;                   /* CG_MAXITER     (src/plugin.cc:241) */
    int maxiter;                      /* MAXITER        (src/plugin.cc:100) */
} v2b_sdp_options;

/* libsdp::SDPCallbackFunction: out = A.in or A^T.in; the callee overwrites out */
typedef void (*v2b_sdp_callback)(double *out, double *in, void *data);
/* libsdp::SDPProgressMonitorFunction (src/v2rdm_casscf/v2rdm_solver.cc:115-124) */
typedef void (*v2b_sdp_monitor)(int print_level, int oiter, int iiter, double energy_primal,
                                double energy_dual, double mu, double primal_error,
                                double dual_error, void *data);

typedef struct v2b_bpsdp v2b_bpsdp;
typedef struct v2b_problem v2b_problem;

const char *v2b_last_error(void);
int v2b_version(void);

/* ---- 1. libsdp-shaped solver ------------------------------------------------ */

/* replaces libsdp::BPSDPSolver(long n_primal, long n_dual, SDPOptions)
 * (src/v2rdm_casscf/v2rdm_solver.cc:433) */
int v2b_bpsdp_create(long n_primal, long n_dual, const v2b_sdp_options *options,
                     v2b_bpsdp **out);
/* replaces BPSDPSolver::solve(x, b, c, primal_block_dims, maxiter, Au, ATu,
 * monitor, print_level, data) (src/v2rdm_casscf/v2rdm_solver.cc:1340).
 * x is updated in place; mu, y, z persist across calls.  Returns V2B_OK when
 * converged, V2B_NOT_CONVERGED when maxiter iterations ran without converging. */
int v2b_bpsdp_solve(v2b_bpsdp *s, double *x, const double *b, const double *c,
                    const int *primal_block_dims, int n_blocks, int maxiter,
                    v2b_sdp_callback Au, v2b_sdp_callback ATu, v2b_sdp_monitor monitor,
                    int print_level, void *data);
/* SDPSolver::is_converged() (src/v2rdm_casscf/v2rdm_solver.cc:1361) */
int v2b_bpsdp_is_converged(const v2b_bpsdp *s);
/* SDPSolver::get_mu / set_mu (src/v2rdm_casscf/v2rdm_solver.cc:1323) */
double v2b_bpsdp_get_mu(const v2b_bpsdp *s);
int v2b_bpsdp_set_mu(v2b_bpsdp *s, double mu);
/* SDPSolver::get_y / get_z copy out; set_y / set_z copy in
 * (src/v2rdm_casscf/checkpoint.cc:58-120) */
int v2b_bpsdp_get_y(const v2b_bpsdp *s, double *y);
int v2b_bpsdp_get_z(const v2b_bpsdp *s, double *z);
int v2b_bpsdp_set_y(v2b_bpsdp *s, const double *y);
int v2b_bpsdp_set_z(v2b_bpsdp *s, const double *z);
/* SDPSolver::iiter_total / oiter_total (src/v2rdm_casscf/v2rdm_solver.cc:1546-1547) */
long v2b_bpsdp_iiter_total(const v2b_bpsdp *s);
long v2b_bpsdp_oiter_total(const v2b_bpsdp *s);
void v2b_bpsdp_destroy(v2b_bpsdp *s);

/* ---- 2. device-map problems -------------------------------------------------- */

/* Sets up the C1 problem that v2RDMSolver::initialize_common_elements builds
 * (src/v2rdm_casscf/v2rdm_solver.cc:1087-1107: set_constraints,
 * build_mapping_arrays, determine_n_primal/dual, set_primal_offsets) for nmo
 * active orbitals, nalpha/nbeta electrons and the POSITIVITY / CONSTRAIN_SPIN /
 * CONSTRAIN_SZ options; hubbard_multiplicity selects the 2S+1 convention of
 * the Hubbard initialiser (v2rdm_solver.cc:862) over the external one (:983). */
int v2b_problem_create(int nmo, int nalpha, int nbeta, int positivity, int constrain_spin,
                       int constrain_sz, int hubbard_multiplicity, v2b_problem **out);
/* The v2RDM-DOCI program that v2RDM_DOCISolver::common_init sets up
 * (src/v2rdm_doci/v2rdm_doci_solver.cc:427-700: POSITIVITY D ... DQGT1T2 and
 * CONSTRAIN_D3, C1, no frozen or restricted orbitals), as a problem for the
 * same v2b_problem_* calls: b (BuildConstraints, :1338-1507), c from h and
 * (ij|kl) (RepackIntegrals, tei.cc:127-153), the random guess (:1325-1336),
 * A.x and A^T.y (bpsdp_Au / bpsdp_ATu, :1509-1566) and the solves.
 * positivity = V2B_POSITIVITY_* | V2B_CONSTRAIN_D3.  DOCI has no Hubbard c
 * and no HF guess: those calls return V2B_BAD_ARG.
 * v2b_problem_pack_spatial_density packs a DOCI solution as hilbert's DOCI
 * PackSpatialDensity does (v2rdm_doci_solver.cc:1568-1703). */
int v2b_doci_problem_create(int nmo, int nalpha, int nbeta, int positivity, v2b_problem **out);
/* A DOCI primal vector (host) in the v2RDM spin-block layout that hilbert's
 * DOCI PackSpatialDensity builds first (v2rdm_doci_solver.cc:1570-1597):
 * D2ab (gab^2, gab = nmo^2), D2aa and D2bb (gaa^2 each, gaa = nmo(nmo-1)/2,
 * D2bb = D2aa), D1a and D1b (nmo^2 each, diagonal), geminals numbered as
 * v2b_problem_create numbers them.  *size receives the length; out may be
 * NULL to ask for it. */
int v2b_doci_v2rdm_layout(const v2b_problem *p, const double *x, double *out, long *size);
/* Independent problems (count >= 1, each from v2b_problem_create or
 * v2b_doci_problem_create) as one problem whose every device launch covers
 * them all: x, b, c and y are the parts' vectors concatenated in order, the
 * PSD blocks the parts' blocks in order, and A is block diagonal.  The joint
 * boundary-point SDP separates into the parts, so a solve converges to the
 * parts' own optima side by side (the penalty mu, the CG scalars and the
 * convergence test are shared).  No counterpart in the reference, which
 * solves one problem per call.  V2B_BAD_ARG when the parts' coefficients do
 * not fit one 16-entry palette.  The parts may be destroyed afterwards.
 * build_b, build_c_*, guess, the density packing and the RDM records are
 * the parts' own: they return V2B_BAD_ARG on a batch. */
int v2b_batch_problem_create(const v2b_problem *const *parts, int count, v2b_problem **out);
/* The distinct coefficients of A (transposed = 0) or A^T (1), at most 16:
 * *count receives how many; out (may be NULL) the values.  Parts whose
 * palettes together hold at most 16 values can share one batch. */
int v2b_problem_palette(const v2b_problem *p, int transposed, double *out, int *count);
void v2b_problem_destroy(v2b_problem *p);
long v2b_problem_n_primal(const v2b_problem *p);
long v2b_problem_n_dual(const v2b_problem *p);
int v2b_problem_n_blocks(const v2b_problem *p);
/* dimensions_ (v2rdm_solver.cc:3729-4079) */
int v2b_problem_block_dims(const v2b_problem *p, int *dims);
/* BuildConstraints (v2rdm_solver.cc:1826-2992) */
int v2b_problem_build_b(const v2b_problem *p, double *b);
/* c for the 1D Hubbard ring (oei.cc:76-95, tei.cc:285-292) */
int v2b_problem_build_c_hubbard(const v2b_problem *p, double t, double U, double *c);
/* c for an external Hamiltonian (v2rdm_solver.cc:147-195): h[nmo^2], g[nmo^4] = (ij|kl) */
int v2b_problem_build_c_external(const v2b_problem *p, const double *h, const double *g,
                                 double *c);
/* Guess (v2rdm_solver.cc:1711-1824): hf = 0 random (srand(0)), hf = 1 HF determinant */
int v2b_problem_guess(const v2b_problem *p, int hf, double *x);
/* bpsdp_Au / bpsdp_ATu (v2rdm_solver.cc:2995-3108) on DEVICE pointers, on
 * the given cudaStream_t (0 = legacy default stream) */
int v2b_problem_Au(v2b_problem *p, const double *d_in, double *d_out, void *stream);
int v2b_problem_ATu(v2b_problem *p, const double *d_in, double *d_out, void *stream);
/* Per-block PSD projection on DEVICE pointers: x = U+ / mu, z = U+ - sym(U),
 * one block per entry of the problem's block_dims. */
int v2b_problem_project(v2b_problem *p, const double *d_U, double mu, double *d_x, double *d_z,
                        void *stream);
/* No counterpart in the reference.  Like v2b_problem_project, but each block
 * starts from the eigenvector basis that the previous warm projection or
 * device solve of this problem left (the identity after creation or after a
 * v2b_problem_project call), as every iteration of the device solve does. */
int v2b_problem_project_warm(v2b_problem *p, const double *d_U, double mu, double *d_x, double *d_z,
                             void *stream);
/* Runs the outer protocol of v2RDMSolver::compute_energy for Hubbard /
 * external Hamiltonians (v2rdm_solver.cc:1296-1361): repeated solve() calls
 * of mu_update_frequency iterations, mu <- mu*eps_p/eps_d between calls,
 * until converged or options->maxiter outer iterations.  x (in/out), b, c are
 * host arrays.  On return *oiter / *iiter hold the iteration totals and
 * *energy the primal energy c.x. */
int v2b_problem_solve(v2b_problem *p, double *x, const double *b, const double *c,
                      const v2b_sdp_options *options, int mu_update_frequency,
                      v2b_sdp_monitor monitor, int print_level, void *data, long *oiter,
                      long *iiter, double *energy);
/* Same iteration with x, b, c already in device memory (x updated in place). */
int v2b_problem_solve_device(v2b_problem *p, double *d_x, const double *d_b, const double *d_c,
                             const v2b_sdp_options *options, int mu_update_frequency,
                             v2b_sdp_monitor monitor, int print_level, void *data, long *oiter,
                             long *iiter, double *energy);
/* dual variables and penalty of the last device solve (host copies) */
int v2b_problem_get_y(const v2b_problem *p, double *y);
int v2b_problem_get_z(const v2b_problem *p, double *z);
double v2b_problem_get_mu(const v2b_problem *p);
/* Restart from a checkpoint (ReadFromCheckpointFile,
 * src/v2rdm_casscf/checkpoint.cc:90-124: MU, DUAL 1 = y, DUAL 2 = z; PRIMAL
 * is the solve's own x argument): the next v2b_problem_solve or
 * v2b_problem_solve_device starts from mu > 0, y (n_dual) and z (n_primal)
 * instead of mu = 0.1 and y = z = 0.  Host arrays, copied here; one solve
 * uses them. */
int v2b_problem_set_state(v2b_problem *p, double mu, const double *y, const double *z);
/* No counterpart in the reference (its solver has no device waits).  The
 * conjugate-gradient kernel is one persistent launch whose blocks meet at
 * grid barriers; each wait polls at most `polls` times (32 ns sleeps between
 * polls) before it records V2B_DEVICE_TIMEOUT, every block leaves at its next
 * barrier and the solve returns that status.  0 restores the default of 40
 * million polls (seconds).  The device solve also checks x, b and c for
 * non-finite values before its first iteration and returns V2B_NAN, naming
 * the vector and index, without iterating (v2b_problem_solve checks the host
 * arrays before any device work). */
int v2b_problem_set_wait_limit(v2b_problem *p, long long polls);
/* libsdp's solver keeps mu, y and z from one solve() call to the next, and
 * hilbert's orbital-optimising loops rely on it: solve(ORBOPT_FREQUENCY),
 * rotate the orbitals (new c), solve again from where the SDP stopped
 * (src/v2rdm_casscf/v2rdm_solver.cc:1330-1361,
 * src/v2rdm_doci/v2rdm_doci_solver.cc:1111-1137).  A device solve starts
 * from mu = 0.1 and y = z = 0 unless this is called before it: then the next
 * v2b_problem_solve or v2b_problem_solve_device continues from the mu, y, z
 * and eigenvector bases that the last device solve of p left (x is the
 * solve's own argument).  V2B_BAD_ARG before the first device solve. */
int v2b_problem_continue(v2b_problem *p);
/* The packed constraint operator the device maps read: A (transposed = 0,
 * rows = dual constraints) or A^T (transposed = 1, rows = primal elements).
 * Entry bits 0..26 hold the column, 27..30 an index into the palette of
 * coefficients, bit 31 marks terms summed into the row's second partial sum
 * (q2.cc:218-318).  Terms are stored in hilbert's accumulation order. */
int v2b_problem_operator_size(const v2b_problem *p, int transposed, long *nrows, long *nnz,
                              int *npalette);
int v2b_problem_operator(const v2b_problem *p, int transposed, uint32_t *row_ptr,
                         uint32_t *entries, double *palette);
/* number of kernels the library launched since the problem was created */
long v2b_problem_kernel_launches(const v2b_problem *p);
/* CUDA-event timing of each kernel class of the device iteration, recorded on
 * the library's stream: 0 cg_kernel, 1 spmv_AT_U_kernel, 2 jacobi_project_kernel,
 * 3 spmv_A2_kernel, 4 stats_kernel.  set_profiling resets the totals; on =
 * 0 off, 1 the kernel classes only, 2 also the phases below (the CG kernel's
 * phase clock and the projection's per-phase events cost some time). */
int v2b_problem_set_profiling(v2b_problem *p, int on);
/* with profiling level 2: CUDA-event time of the projection's phases, the first
 * count of: [0] GEMM tiles, [1] acceptance test, [2] clusters + Newton step,
 * [3] block-Jacobi sweeps, [4] Jacobi kernels (no reference counterpart) */
int v2b_problem_projection_profile(const v2b_problem *p, double *ms, long *n, int count);
/* with profiling level 2: milliseconds of the CG kernel's phases, barrier to
 * barrier on the kernel's own clock, the first count of: [0] initial
 * residual, [1] the new direction p, t = A^T p and ||t||^2, [2] A t with the
 * y and r update and r.r, [3] zero (no reference counterpart) */
int v2b_problem_cg_profile(const v2b_problem *p, double *ms, int count);
int v2b_problem_profile(const v2b_problem *p, double *ms /* [5] */, long *launches /* [5] */);
/* the cudaStream_t the device solve runs on (after the first device call) */
void *v2b_problem_stream(const v2b_problem *p);
/* projection work since the last reset: warm-started calls, Jacobi rotations
 * applied, and blocks whose Jacobi sweeps hit the sweep cap */
int v2b_problem_projection_counts(const v2b_problem *p, long *calls, long *rotations,
                                  long *sweep_overruns);
/* No counterpart in the reference (libsdp diagonalises every block with LAPACK
 * each iteration).  Warm refinement of the projection since the problem was
 * created, the first n of: [0] blocks accepted without Jacobi, [1] blocks
 * projected by the Jacobi kernels, [2] acceptance tests run (one per pass and
 * call), [3] clusters diagonalised exactly, [4] blocks that changed to
 * block-Jacobi sweeps for a cluster above 64 rows, [5] ... for too many
 * non-separable pairs, [6] blocks handed to the Jacobi kernels after their
 * passes or sweeps ran out, [7] block-Jacobi sweeps run, [8] FP32
 * eigensolves of blocks (projection mode 2). */
int v2b_problem_refine_counts(const v2b_problem *p, long *counts, int n);
/* No counterpart in the reference.  Projection method of the device solve:
 * 0 (default) warm refinement with block-Jacobi and Jacobi fallbacks; 1 the
 * plain path, selective Jacobi on every block in every iteration (the
 * per-iteration full eigendecomposition libsdp performs, in FP64); 2 mixed
 * precision: warm refinement in which a block above 160 rows that would
 * change to block-Jacobi sweeps first takes an FP32 selective Jacobi
 * eigensolve (FP32 storage and updates, FP64 rotations), then an FP64
 * Rayleigh-Ritz step (T recomputed in the new basis) and the FP64
 * acceptance test and Newton passes. */
int v2b_problem_set_projection_mode(v2b_problem *p, int mode);

/* The projection's FP64 GEMM launches cut the K range of large blocks' tiles
 * into parts (the count chosen by a timed autotuner when the plan is
 * built), and sum the parts in a fixed order (run-to-run identical).  on = 0
 * computes every tile in one piece.  Default on.  No reference counterpart: libsdp
 * projects with LAPACK on the host. */
int v2b_problem_set_gemm_split(v2b_problem *p, int on);
/* The part counts S the split autotuner chose when the projection plan was
 * built (the first projection): for the full tile list (W = Us Vt^T) and for
 * the upper-tile list of the symmetric products (T = Vt W, U+ = Vt^T P Vt).
 * Each is the fastest of S = 1, 2, 4 in timed launches over every block on
 * this GPU; 0 before the plan exists. */
int v2b_problem_gemm_split_choice(const v2b_problem *p, int *full, int *upper);

/* ---- 2b. densities for the orbital optimiser --------------------------------- */

/* PackSpatialDensity (v2rdm_solver.cc:3110-3219, C1): from a primal x on the
 * device, the spin-summed active 2-RDM packed over the n(n+1)/2 symmetric
 * geminals (lower triangle of geminal pairs, off-diagonal pairs doubled;
 * d2_size = g00 (g00 + 1) / 2, g00 = n (n + 1) / 2) and the spin-summed 1-RDM
 * (lower triangle, d1_size = g00), bit-identical to hilbert's. */
int v2b_problem_pack_dims(const v2b_problem *p, long *d2_size, long *d1_size);
int v2b_problem_pack_spatial_density(v2b_problem *p, const double *d_x, double *d_d2, double *d_d1,
                                     void *stream);

/* The density-matrix records hilbert writes after a solve, from the host
 * primal vector x: the same records, order and values as WriteTPDM
 * (src/v2rdm_casscf/write_tpdm.cc:40-310: files D2aa, D2bb, D2ab),
 * WriteTPDMSpinFree (:312-519: file D2) and WriteOPDM (write_opdm.cc:40-114:
 * files D1a, D1b), for C1 with ncore >= 0 doubly occupied (restricted)
 * orbitals numbered 0 .. ncore-1 ahead of the active ones (active orbital i
 * is ncore + i), including the writers' core-core and core-active records.  The record layouts are the reference's struct
 * tpdm and struct opdm (v2rdm_solver.h:53-65).  counts[6] receives the
 * record counts in the order D2aa, D2bb, D2ab, D2, D1a, D1b, -1 for a file
 * the problem's writers do not write: a DOCI problem gives what v2RDM-DOCI's
 * WriteTPDM writes (src/v2rdm_doci/write_tpdm.cc:47-176: D2aa, D2bb, D2ab
 * only).  Any output array may be NULL. */
typedef struct {
    int i, j, k, l;
    double value;
} v2b_tpdm_record;
typedef struct {
    int i, j;
    double value;
} v2b_opdm_record;
int v2b_problem_rdm_counts(const v2b_problem *p, int ncore, long *counts);
int v2b_problem_rdm_records(const v2b_problem *p, int ncore, const double *x, v2b_tpdm_record *d2aa,
                            v2b_tpdm_record *d2bb, v2b_tpdm_record *d2ab, v2b_tpdm_record *d2,
                            v2b_opdm_record *d1a, v2b_opdm_record *d1b);
/* The 2-RDM as WriteTPDM_IWL hands it to Psi4's IWL writer for gradients
 * (src/v2rdm_casscf/write_tpdm_iwl.cc:45-205): one record per write_value
 * call, in call order, labels (i, k, j, l) for the element D2(ij, kl), aa and
 * bb values scaled by 1/4, core orbitals as in v2b_problem_rdm_records
 * (record counts: counts[0] and counts[2] of v2b_problem_rdm_counts).  The IWL files store only values above their
 * cutoff, 1e-14; that filtering is the IWL writer's.  v2RDM problems only. */
int v2b_problem_tpdm_iwl_records(const v2b_problem *p, int ncore, const double *x, v2b_tpdm_record *d2aa,
                                 v2b_tpdm_record *d2ab, v2b_tpdm_record *d2bb);
/* The 3-RDM records of WriteActive3PDM (src/v2rdm_casscf/write_3pdm.cc:50-206;
 * 3PDM_WRITE with CONSTRAIN_D3), files D3aaa, D3aab, D3bba, D3bbb, layout
 * struct dm3 (:39-47), orbitals numbered as in v2b_problem_rdm_records.
 * counts[0]: records in D3aaa and in D3bbb; counts[1]: in D3aab and D3bba.
 * Problems with the D3 blocks only. */
typedef struct {
    int i, j, k, l, m, n;
    double value;
} v2b_dm3_record;
int v2b_problem_d3_counts(const v2b_problem *p, long *counts);
int v2b_problem_d3_records(const v2b_problem *p, int ncore, const double *x, v2b_dm3_record *d3aaa,
                           v2b_dm3_record *d3aab, v2b_dm3_record *d3bba, v2b_dm3_record *d3bbb);

/* ---- 2c. the orbital step's integral transform -------------------------------- */

/* focas's density-fitted integral transform (OrbitalOptimizer::TransformTei_Q,
 * src/focas/C_files/orbopt_integraltransform_cpu.cc:235-261, and
 * TransformOei, :263-285, for count = 1): d_Bp[Q] = U^T d_B[Q] U for
 * Q = 0 .. count-1, n x n row-major matrices in device memory, on FP64
 * tensor cores, one matrix per CTA.  n <= 80, else V2B_BAD_ARG. */
int v2b_df_transform(const double *d_U, const double *d_B, double *d_Bp, int n, int count, void *stream);
/* No counterpart in the reference (focas has no derivative with respect to
 * U).  The adjoint of the transform: d_dU = sum_Q (B_Q U M_Q^T + B_Q^T U M_Q),
 * the gradient of sum_Q <M_Q, U^T B_Q U> with respect to U, summed over Q in
 * order.  d_work: count * n * n doubles of scratch.  n <= 80. */
int v2b_df_transform_adjoint(const double *d_U, const double *d_B, const double *d_M, double *d_dU,
                             double *d_work, int n, int count, void *stream);

/* ---- 3. allocation-free projection ------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need a projection (their host owns all device memory, or the
 * device synchronisation of an allocation is not acceptable there): projects
 * ONE n x n block d_U (row-major, device memory) like v2b_problem_project,
 * writing d_x = U+ / mu and d_z = U+ - sym(U), on the given cudaStream_t.
 * n <= 128: all scratch is a fixed file-scope device array (about 4.4 MB,
 * held by every GPU that loads the library until exit); larger n returns
 * V2B_BAD_ARG.  Allocates nothing.  Every call reuses the same array, so calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * first call on a device looks the array up with cudaGetSymbolAddress (a
 * call in a new context, after cudaDeviceReset, looks it up again); make it
 * before any stream capture. */
int v2b_project_block_noalloc(const double *d_U, int n, double mu, double *d_x, double *d_z,
                              void *stream);

#ifdef __cplusplus
}
#endif

#endif /* V2RDM_B200_H */
