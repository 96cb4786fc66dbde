/*
 * qd.h -- C ABI of the B200 split-operator wavepacket propagator.
 *
 * The propagator advances a wavepacket psi(R, r, theta) of an atom + diatom
 * system in reactant Jacobi coordinates with the split-operator scheme
 *
 *     psi <- dump * B * Rot(dt/2) * IFFT * T(dt) * FFT * Rot(dt/2) * F * V(dt) * psi
 *
 * (F/B = forward/backward Gauss-Legendre transform theta <-> l, T = radial
 * kinetic phase, Rot = rotational phase, V = potential phase, dump = absorber)
 * and accumulates the flux through a dividing surface r = r_s into
 * initial-state-selected reaction probabilities P(E).
 *
 * The structs below carry exactly the fields of the Matlab struct that the
 * reference MEX entry point reads (common/MatlabStructures.h:12-157,
 * common/MatlabStructures.C:17-97, common-cuda/MatlabStructures.h:100), with the
 * same names, units (bohr, hartree, atomic time, electron masses) and memory
 * layouts:
 *   psi, pot : column-major n1 x n2 x n_theta, index (k*n2 + j)*n1 + i,
 *              psi complex128 interleaved (re, im), pot real double;
 *   theta.legendre : (m+1) x n column-major, P_l(x_k) at [l + k*(m+1)].
 * Arrays are owned by the caller; psi, time.steps and CRP.CRP are updated in
 * place, as the reference does with Matlab-owned memory.
 *
 * Every function returns an int status: QD_OK (0) or a negative QD_ERR_* code;
 * qd_last_error() returns the message of the last failure on the calling
 * thread.  Nothing longjmps or throws across this boundary.
 */
#ifndef QD_H
#define QD_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QD_ABI_VERSION 2

/* status codes */
#define QD_OK               0
#define QD_ERR_INVALID     -1  /* bad argument / inconsistent sizes          */
#define QD_ERR_CUDA        -2  /* CUDA runtime or driver error                */
#define QD_ERR_NOMEM       -3  /* host or device allocation failed            */
#define QD_ERR_PES         -4  /* PES callback returned non-zero or non-finite*/
#define QD_ERR_NONFINITE   -5  /* NaN/Inf or norm growth detected in psi      */
#define QD_ERR_UNSUPPORTED -6  /* size/option not supported by the kernels    */
#define QD_ERR_IO          -7  /* file read/write error (.grids, checkpoint)  */
#define QD_ERR_DEVICE      -8  /* device-side status word reported a failure  */
#define QD_ERR_STOPPED     -9  /* a progress callback asked to stop           */

/* arithmetic of the propagation */
#define QD_PREC_FP64  0  /* plain form: complex128 psi, FP64 everywhere       */
#define QD_PREC_FP32  1  /* complex64 psi, 3xFP16 tensor-core Legendre GEMM,
                            FP64 flux-to-P(E) accumulation and norm; the
                            input psi is rounded to complex64 when the handle
                            is created (it crosses the bus in complex64), and
                            psi read back is that complex64 state, widened  */

/* RadialCoordinate (common/MatlabStructures.h:12-39).  r0, k0, delta are the
 * initial-packet parameters that only the setup helpers read
 * (H3/InitWavePacket.m:8-13, common/EtaSq.m:3-5). */
typedef struct qd_radial {
  int32_t       n;
  const double *r;      /* n grid points, uniform spacing dr            */
  double        dr;
  double        mass;   /* reduced mass in electron masses              */
  double        r0, k0, delta;
} qd_radial;

/* AngleCoordinate (common/MatlabStructures.h:41-66). */
typedef struct qd_angle {
  int32_t       n;        /* number of Gauss-Legendre points n_theta    */
  int32_t       m;        /* highest Legendre order; n_l = m + 1        */
  const double *x;        /* cos(theta_k), n                            */
  const double *w;        /* quadrature weights, n                      */
  const double *legendre; /* (m+1) x n, P_l(x_k) at [l + k*(m+1)]       */
} qd_angle;

/* EvolutionTime (common/MatlabStructures.h:68-90).  steps is in/out: a call
 * with steps == 0 applies the V(-dt/2) pre-step first (timeEvol.C:664-665). */
typedef struct qd_time {
  int32_t total_steps;
  double  time_step;
  int32_t steps;
} qd_time;

/* The C ABI counterpart of options.wave_to_matlab (common/wave2matlab.C:26-34,
 * common-cuda/evolutionCUDA2.cu:540-546).  qd_time_evolution /
 * qd_time_evolution_batch call it whenever time.steps reaches a multiple of
 * steps_to_copy_psi_from_device_to_host, after writing that step's psi (the
 * caller's array, passed again as `psi`), time.steps and CRP.CRP into the
 * run's struct; `norm` is the run's wavepacket norm after the step.  Return
 * 0 to continue, non-zero to stop the call with QD_ERR_STOPPED (the struct
 * then holds the state of that step). */
typedef int (*qd_progress_fn)(int32_t step, double norm, const double *psi,
                              void *ctx);

/* Options (common/MatlabStructures.h:92-113; the CUDA variant adds
 * steps_to_copy_psi_from_device_to_host, common-cuda/MatlabStructures.h:100). */
typedef struct qd_options {
  const char    *wave_to_matlab;  /* kept for schema parity; not executed   */
  const char    *test_name;
  /* N > 0: every N steps (time.steps % N == 0) qd_time_evolution writes psi,
   * time.steps and CRP.CRP back and calls progress (the reference's GPU loop
   * computes P(E) and copies psi back on those steps); 0 = only at the end */
  int32_t        steps_to_copy_psi_from_device_to_host;
  int32_t        precision;       /* QD_PREC_FP64 (default) or QD_PREC_FP32 */
  qd_progress_fn progress;        /* optional                               */
  void          *progress_ctx;
} qd_options;

/* DumpFunction (common/MatlabStructures.h:115-129).  NULL = absent; the
 * absorber is applied only when both dump1 and dump2 are present
 * (timeEvol.h:117). */
typedef struct qd_dump {
  const double *dump;
} qd_dump;

/* CummulativeReactionProbabilities (common/MatlabStructures.h:131-157).
 * n_dividing_surface is a 1-based r2 index (Gradient3.F:45). */
typedef struct qd_crp {
  int32_t       n_dividing_surface;
  int32_t       n_gradient_points;  /* odd, 3..11 (Gradient3.F:14-26)        */
  int32_t       n_energies;
  int32_t       calculate_CRP;
  const double *energies;           /* hartree, n_energies                   */
  const double *eta_sq;             /* n_energies                            */
  double       *CRP;                /* out: P(E), n_energies                 */
} qd_crp;

/* Centrifugal-sudden block (J, K).  No counterpart in the reference, whose
 * propagator is the J = 0 one; zero-initialised it is exactly that.  For a
 * block (J, K) the angular basis is the normalised associated Legendre
 * functions of order K, j = K .. K + m: theta.legendre holds
 * L[l][k] = Pbar_{K+l}^K(x_k) / sqrt(l + 1/2) (so the reference's transform
 * pair, B with L and F with (l+1/2) w_k L, stays an identity on the basis;
 * qd_cs_legendre builds it), the rotational phase uses j(j+1) with j = K + l,
 * and pot already contains the centrifugal term (J(J+1) - 2K^2)/(2 mu_R R^2)
 * (the caller's to add, as it adds any potential). */
typedef struct qd_cs {
  int32_t J;
  int32_t K;
} qd_cs;

/* The whole Matlab struct handed to TimeEvolutionMex / TimeEvolutionMexCUDA
 * (common/TimeEvolutionMex.C:28-70), followed by the centrifugal-sudden block
 * indices (zero for the reference's J = 0 propagation). */
typedef struct qd_data {
  qd_radial   r1;       /* R, atom - diatom distance                         */
  qd_radial   r2;       /* r, diatom bond length                             */
  qd_angle    theta;
  const double *pot;    /* n1*n2*n_theta hartree                             */
  double     *psi;      /* n1*n2*n_theta complex128 interleaved, in/out      */
  qd_time     time;
  qd_options  options;
  qd_dump     dump1, dump2;
  qd_crp      CRP;
  qd_cs       cs;
} qd_data;

/* ---- library ---------------------------------------------------------- */

int         qd_abi_version(void);
const char *qd_last_error(void);
/* Number of CUDA kernel launches issued by this library in this process. */
int64_t     qd_kernel_launch_count(void);
/* Select the CUDA device that later calls on this thread use (the library
 * links the CUDA runtime statically, so the caller's own runtime device
 * choice does not carry over). */
int         qd_set_device(int32_t device);

/* Drop-in for the MEX entry point TimeEvolutionMexCUDA(struct)
 * (common-cuda/TimeEvolutionMexCUDA.C:20-83, CPU twin
 * common/TimeEvolutionMex.C:18-78): uploads pot and psi, propagates
 * data->time.total_steps steps on device 0 of the calling thread, writes psi,
 * time.steps and (if CRP.calculate_CRP) CRP.CRP back in place.  As in the
 * reference, the flux accumulators start from zero at every call. */
int qd_time_evolution(qd_data *data);

/* ---- handle API: device-resident state across calls -------------------- */

typedef struct qd_handle qd_handle;

/* Validate data, build all tables on the device and upload psi.  data's
 * arrays must stay valid until qd_destroy (psi/CRP are written back by
 * qd_download / qd_get_crp). */
int qd_create(const qd_data *data, qd_handle **out);
int qd_destroy(qd_handle *h);
/* Propagate n_steps steps (device-resident; no host copies). */
int qd_propagate(qd_handle *h, int32_t n_steps);
/* qd_propagate that also reports the device time of the n_steps steps
 * (CUDA events on the handle's stream, summed over steps).  If
 * flush_bytes > 0 a buffer of that size is overwritten and then read back
 * between steps, outside the timed spans, so that every step starts with a
 * cold L2 (holding none of the propagation's data and no dirty lines). */
int qd_propagate_timed(qd_handle *h, int32_t n_steps, int64_t flush_bytes,
                       double *device_ms);
/* Current theta-space psi (layout of qd_data.psi) into psi_out (host). */
int qd_get_psi(qd_handle *h, double *psi_out);
/* Current P(E) (CRPAux.F:34-66 applied to the accumulated phi_E, dphi_E). */
int qd_get_crp(qd_handle *h, double *crp_out);
/* Copy psi, time.steps and CRP back into the qd_data given to qd_create. */
int qd_download(qd_handle *h);
/* Wavepacket norm after each propagated step (FP64, module_for_psi,
 * timeEvol.C:220-243); norms_out holds n entries, oldest first, ending at the
 * last step.  n <= steps propagated by this handle. */
int qd_get_norms(qd_handle *h, double *norms_out, int32_t n);
/* Kinetic, rotational, potential and total energy of the current psi
 * (timeEvol.C:256-283, 323-360, 390-436), hartree. */
int qd_energies(qd_handle *h, double out4[4]);
/* Energies inside the propagation, the reference's per-step diagnostics
 * (potential_energy, rotational_energy, kinetic_energy_for_legendre_psi;
 * timeEvol.C:256-283, 323-360, 390-436) at an interval: with every > 0, on
 * each step whose count time.steps is a multiple of `every`, the step's own
 * kernels add FP64 partial sums (kinetic and rotational in the l-space pass,
 * potential in the column pass that forms that step's theta-space
 * wavepacket), copied back once per qd_propagate call.  0 turns it off
 * (the default). */
int qd_set_energy_interval(qd_handle *h, int32_t every);
/* The newest min(cap, recorded) energy records of one run, oldest first, five
 * doubles each: step, E_kin, E_rot, E_pot, E_total (hartree); n_out = records
 * written. */
int qd_get_energy_log_run(qd_handle *h, int32_t run, double *out, int32_t cap, int32_t *n_out);
/* Steps propagated so far (the handle's time.steps). */
int qd_steps(qd_handle *h, int32_t *steps_out);
/* Average device time per step (ms) of each kernel class over the last
 * qd_propagate call when profiling is enabled via qd_set_profiling(h, 1). */
int qd_set_profiling(qd_handle *h, int32_t on);
int qd_kernel_times(qd_handle *h, double *ms_out, int32_t n, int32_t *n_written);
/* The kernels this handle's autotuners picked (the choice is kept per shape
 * for the process): out[0] = the complex64 l-space kernel (0 the split row and
 * column kernels, 1/2/4 the Stockham cluster kernel on that many CTAs per
 * slice, 8/9/10 the register-FFT kernel on 1/2/4 CTAs per slice, 11 its 4-CTA
 * form with 16 x 16 row transforms; 0 for the FP64 form), out[1] = 1 if the
 * column pass runs on the tensor cores, out[2] = the flux-accumulation GEMM
 * tile variant (0-3), out[3] = 1 if full 250-step chunks of flux history are
 * accumulated in the chirp-z form (energies on a uniform grid). */
int qd_kernel_choice(qd_handle *h, int32_t out[4]);

/* Checkpoint / restart of the full propagation state: the l-space
 * wavepacket, time.steps, the flux accumulators phi_E, dphi_E and the
 * pending flux history, and the per-step norms.  The reference keeps only psi
 * and time.steps across calls (timeEvol.C:664-665), so its P(E) restarts;
 * qd_restore resumes the accumulation exactly.  qd_restore needs a handle
 * created from data of the same sizes and precision. */
int qd_checkpoint(qd_handle *h, const char *path);
int qd_restore(qd_handle *h, const char *path);

/* ---- batches: many propagations in the same launches ------------------- */

/* runs[0..n_runs) share r1, r2, theta.n/x/w, time.time_step, time.steps,
 * options.precision, the absorbers and the CRP settings (surface, stencil,
 * number of energies); psi, pot, theta.m/legendre, cs, CRP.energies and
 * CRP.eta_sq may differ per run (one potential table is kept when all pot
 * arrays are equal; runs with fewer angular functions are padded with empty
 * l-slices).  All runs
 * advance together; results per run.  No counterpart in the reference, whose
 * MEX propagates one wavepacket per call. */
int qd_create_batch(const qd_data *runs, int32_t n_runs, qd_handle **out);
int qd_time_evolution_batch(qd_data *runs, int32_t n_runs);
int qd_n_runs(qd_handle *h, int32_t *n_out);
int qd_get_psi_run(qd_handle *h, int32_t run, double *psi_out);
int qd_get_crp_run(qd_handle *h, int32_t run, double *crp_out);
int qd_get_norms_run(qd_handle *h, int32_t run, double *norms_out, int32_t n);
int qd_energies_run(qd_handle *h, int32_t run, double out4[4]);

/* ---- energies without allocation ----------------------------------------
 * No counterpart in the reference.  Same result as qd_energies_run, but the
 * kinetic-energy DFT scratch (n1*n2*n_theta complex128 values) and the three
 * FP64 sums live in one static device array instead of cudaMalloc'd memory.
 * It serves callers that cannot allocate device memory at diagnostic time:
 * a host that sized a large batch to fill the device and handed the rest to
 * its own memory pool (a cudaMalloc would fail with out-of-memory in the
 * middle of the run), and monitors that sample energies often while other
 * streams keep working (cudaFree synchronises the whole device, so the
 * allocating call stalls them every time).
 *   - limit: n1*n2*n_theta of one run <= QD_ENERGIES_NOALLOC_MAX_POINTS
 *     (16 MiB of scratch); larger grids get QD_ERR_INVALID and nothing runs;
 *   - the first call on each device looks up the scratch address
 *     (cudaGetSymbolAddress, which may load the module holding the array):
 *     make that first call before any stream capture;
 *   - the scratch is shared by every handle on the device, so calls that
 *     overlap in time (two host threads, or two streams) race on it;
 *   - the sums are cleared on the handle's stream at every call. */
#define QD_ENERGIES_NOALLOC_MAX_POINTS 1048576
int qd_energies_noalloc(qd_handle *h, int32_t run, double out4[4]);

/* ---- setup helpers (the Matlab-side L4 of the reference) --------------- */

/* Gauss-Legendre nodes and weights from a "<n>-LegendreGauss.grids" file in
 * dir (format of the reference's GaussLegendre/<n>-LegendreGauss.grids files, reader
 * common/GaussLegendre2.m:1-31):
 * ceil(n/2) lines "x w" of the non-negative half, mirrored; x ascending. */
int qd_read_grids(const char *dir, int32_t n, double *x, double *w);

/* theta.legendre = P_l(x_k), (m+1) x n column-major, by the three-term
 * recurrence of common/LegendreP2.m:9-21, computed in FP64 on the GPU. */
int qd_legendre_matrix(int32_t n, int32_t m, const double *x, double *legendre);

/* ---- learned PES surrogate ---------------------------------------------- */

/* A small permutation-symmetric MLP in place of a PES routine.  No counterpart
 * in the reference, which evaluates its PES (Fortran/MEX) at every grid point.
 * Features p_ij = exp(-r_ij / 1.5 bohr): (p23, p12 + p13, p12 p13), invariant
 * under exchanging the two diatom atoms, standardised; four dense SiLU layers
 * of width 64; linear scalar output (standardised V).  FP32 weights and
 * accumulation in every product, FP32 Adam.  Trained and evaluated
 * on the GPU by this library's kernels; the plain PES judges it. */
typedef struct qd_mlp qd_mlp;
int     qd_mlp_create(qd_mlp **out, uint64_t seed);      /* He-uniform initial weights */
int     qd_mlp_destroy(qd_mlp *m);
int32_t qd_mlp_n_params(void);
/* FP32 master weights (qd_mlp_n_params floats) and the standardisation
 * (feature means[3], feature stds[3], V mean, V std). */
int qd_mlp_get_params(qd_mlp *m, float *w_out, float norm_out[8]);
int qd_mlp_set_params(qd_mlp *m, const float *w, const float norm[8]);
/* Feature and target standardisation from a training set. */
int qd_mlp_fit_normalisation(qd_mlp *m, int64_t n, const double *r12, const double *r23,
                             const double *r13, const double *V);
/* train_steps > 0: that many Adam steps over the n samples in minibatches of
 * `batch` (in order, wrapping), learning rate decaying geometrically from lr
 * to lr_end; loss_out = mean squared error (standardised V) of the last epoch.
 * train_steps <= 0: no update; loss_out = the loss over all n samples and, if
 * grad_out, its gradient with respect to the FP32 parameters. */
int qd_mlp_train(qd_mlp *m, int64_t n, const double *r12, const double *r23, const double *r13,
                 const double *V, int32_t train_steps, int32_t batch, double lr, double lr_end,
                 float *grad_out, double *loss_out);
/* V (hartree) at n geometries, r_ij in bohr. */
int qd_mlp_eval(qd_mlp *m, int64_t n, const double *r12, const double *r23, const double *r13,
                double *V_out);
/* The surrogate on the Jacobi grid with the mapping, mask and cap of
 * qd_potential_jacobi (H3/H3PESJacobi.m:5-27). */
int qd_mlp_potential(qd_mlp *m, const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                     const double masses[3], double vmax, double rmin, int32_t cap,
                     double *pot_out);

/* theta.legendre of centrifugal-sudden block K: L[l][k] =
 * Pbar_{K+l}^K(x_k) / sqrt(l + 1/2), l = 0..m, with Pbar_j^K the associated
 * Legendre function normalised to one on [-1, 1] (no Condon-Shortley phase),
 * by the standard three-term recurrence in j, one FP64 GPU thread per node.
 * K = 0 gives P_l(x_k), the reference's matrix (as qd_legendre_matrix).
 * QD_ERR_INVALID for a node outside [-1, 1]; QD_ERR_CUDA without a GPU. */
int qd_cs_legendre(int32_t n, int32_t K, int32_t m, const double *x, double *legendre);

/* Initial wavepacket on the GPU in FP64 (H3/InitWavePacket.m:13-31,
 * H3/H2VibRotWaveFunction.m:20-46): the v0-th sinc-DVR eigenstate
 * phi_{v0 j0}(r) of the diatom (v_diatom[r2.n] its potential in hartree, plus
 * j0(j0+1)/(2 mu r^2)), largest component positive, times
 * g(R) = (pi delta^2)^(-1/4) exp(-(R-R0)^2/(2 delta^2) - i k0 R) (R0, k0, delta
 * from r1) and the angular function Pbar_{j0}^K(x_k) (sqrt(j0+1/2) P_{j0} for
 * K = 0; zero if K > j0).  psi_out: complex128 in the layout of qd_data.psi;
 * e_vj_out: the diatom level (hartree); phi_out (optional, r2.n): phi_vj. */
int qd_init_state(const qd_radial *R, const qd_radial *r, const qd_angle *theta, int32_t j0,
                  int32_t v0, int32_t K, const double *v_diatom, double *psi_out,
                  double *e_vj_out, double *phi_out);
/* eta^2(E) of the initial packet (common/EtaSq.m:12-15) at collision
 * energies e_coll (hartree), on the GPU in FP64. */
int qd_eta_sq(const qd_radial *R, int32_t ne, const double *e_coll, double *eta_sq_out);

/* ---- potential on the Jacobi grid (H3/H3PESJacobi.m:5-27) --------------- */

/* A PES in the convention of the reference's PES MEX functions
 * (FH2/HSW/HSWMex.C:29-90, called as H3PES(r12, r23, r13) by
 * H3/H3PESJacobi.m:25): V[m] = V(r12[m], r23[m], r13[m]) for n points,
 * internuclear distances in bohr (atom 1 = the atom, 2 3 = the diatom), V in
 * hartree.  Return 0 on success; any other value aborts with QD_ERR_PES. */
typedef int (*qd_pes_fn)(int64_t n, const double *r12, const double *r23, const double *r13,
                         double *V, void *ctx);

/* pot_out (n1 x n2 x n_theta, the layout of qd_data.pot) on the Jacobi grid
 * R = r1.r, r = r2.r, cos(theta) = theta.x: r23 = r,
 * r12 = sqrt((f2 r)^2 + R^2 - 2 f2 r R cos), r13 = sqrt((f3 r)^2 + R^2 + 2 f3 r R cos),
 * f2 = masses[2]/(masses[1]+masses[2]), f3 = 1 - f2.  Points with any distance
 * <= rmin get vmax; if cap, V is also capped at vmax.  One callback for all
 * other points, on the calling thread. */
int qd_potential_jacobi(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                        const double masses[3], qd_pes_fn pes, void *ctx, double vmax,
                        double rmin, int32_t cap, double *pot_out);

/* Extended-LEPS surface V = De(BC) + Q_AB + Q_BC + Q_AC
 * - sqrt(J_AB^2 + J_BC^2 + J_AC^2 - J_AB J_BC - J_BC J_AC - J_AC J_AB), per pair
 * Q, J = (De (y-2) +- pf (y+2)) y / 2, y = exp(-beta (r - re)),
 * pf = De (1 - sato)/(1 + sato) / 2 (the algebra of ClH2/G3/clh2g3v.F:88-101).
 * No counterpart in the reference's propagator; evaluated on the GPU in FP64. */
typedef struct qd_leps_pair {
  double de;      /* hartree */
  double beta;    /* 1/bohr */
  double re;      /* bohr */
  double sato;
} qd_leps_pair;
typedef struct qd_leps {
  qd_leps_pair ab;  /* atom - diatom atom 2 (r12) */
  qd_leps_pair bc;  /* the diatom (r23)           */
  qd_leps_pair ac;  /* atom - diatom atom 3 (r13) */
} qd_leps;
int qd_potential_leps(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                      const double masses[3], const qd_leps *leps, double vmax, double rmin,
                      int32_t cap, double *pot_out);

/* The BKMP2 surface of H3 (H3/bkmp2.F, Boothroyd-Keogh-Martin-Peterson
 * 1996, the parameter set of that file; replaces the PES MEX
 * H3/BKMP2Mex.C:16-60), evaluated on the GPU in FP64.  qd_bkmp2_eval gives
 * the MEX value (hartree) at n geometries of internuclear distances (bohr);
 * NaN where the reference stops on an impossible triangle or a distance
 * below 0.2 bohr.  qd_potential_bkmp2 fills the Jacobi grid (mapping, mask
 * and cap of qd_potential_jacobi; rmin >= 0.2) with the value minus
 * vH2Min = -0.174495770896975, as H3/H3PESBKMP2.m:23-27 does. */
int qd_bkmp2_eval(int64_t n, const double *r1, const double *r2, const double *r3,
                  double *v_out);
int qd_potential_bkmp2(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                       const double masses[3], double vmax, double rmin, int32_t cap,
                       double *pot_out);

/* The HSW surface of F + H2 (FH2/HSW/hswpot.F:1-99 with sospline.F; replaces
 * the PES MEX FH2/HSW/HSWMex.C:29-90 and its Fortran): the SW1 fit plus the
 * spline-interpolated spin-orbit correction, evaluated on the GPU in FP64.
 * qd_hsw_create reads the reference's own data files three.param, two.param,
 * so.input and so.param from dir (the HSW_DATA_DIR of HSWMex.C:48-56) and
 * builds the spline once on the host; qd_hsw_create_from_tables takes the
 * same numbers as arrays: the three.param records (n3 of them; the last six
 * are b1 b2 b3 x0 y0 z0 in a[]), the 12 two.param values, the so.input grid
 * (nodes x[nx], y[ny], z[nz], values so[i][j][k] in file order, k fastest)
 * and the three so.param values (kcal/mol, bohr, bohr). */
typedef struct qd_hsw qd_hsw;
int qd_hsw_create(const char *dir, qd_hsw **out);
int qd_hsw_create_from_tables(int32_t n3, const int32_t *ix, const int32_t *iy,
                              const int32_t *iz, const double *a, const double p[12],
                              int32_t nx, int32_t ny, int32_t nz, const double *x,
                              const double *y, const double *z, const double *so,
                              const double so_param[3], qd_hsw **out);
int qd_hsw_destroy(qd_hsw *h);
/* V (hartree) at n points given as internuclear distances in bohr, in the
 * argument order of pot() (hswpot.F:1): r(F-H1), r(H1-H2), r(F-H2). */
int qd_hsw_eval(const qd_hsw *h, int64_t n, const double *r_fh1, const double *r_hh,
                const double *r_fh2, double *v_out);
/* The surface on the Jacobi grid, with the mapping, masking and cap of
 * qd_potential_jacobi (atom 1 = F: r12 = r(F-H1), r23 = r(H1-H2), r13 = r(F-H2)). */
int qd_potential_hsw(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                     const double masses[3], const qd_hsw *h, double vmax, double rmin,
                     int32_t cap, double *pot_out);

#ifdef __cplusplus
}
#endif
#endif /* QD_H */
