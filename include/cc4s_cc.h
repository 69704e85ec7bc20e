/* C ABI of the B200 CoupledCluster step (methods Ccsd and Ccd).
 *
 * Drop-in replacement for the cc4s algorithm step
 *   - name: CoupledCluster
 *     in:  {method, slicedEigenEnergies, slicedCoulombVertex, coulombIntegrals,
 *           mixer: {type, maxResidua | ratio}, maxIterations, energyConvergence,
 *           amplitudesConvergence, levelShift, initialAmplitudes,
 *           integralsSliceSize, ppl}
 *     out: {energy: {correlation, direct, exchange, secondOrder, unit},
 *           convergenceReached, amplitudes: {ph, pphh}}
 * The reference binds this step through C++ name registries, not a C ABI:
 *   AlgorithmRegistrar "CoupledCluster"      src/main/algorithms/CoupledCluster.cxx:34-52
 *   CoupledClusterMethodRegistrar "Ccsd"     src/main/algorithms/coupledcluster/Ccsd.cxx:25-32
 *   MixerRegistrar "DiisMixer"/"LinearMixer" src/main/mixers/DiisMixer.cxx:25,
 *                                            src/main/mixers/LinearMixer.cxx:24
 * Each entry point below states the reference interface it replaces.
 *
 * Conventions: every function returns a status (0 = OK).  No C++ exception
 * crosses this boundary; the message of the last failure is available from
 * cc4s_cc_last_error.  Host buffers are owned by the caller and copied; device
 * memory is owned by the handle.  One handle per host thread; each handle
 * owns one CUDA stream.  Tensors use the reference's column-major layout
 * (first index fastest): eps[p], T1[a,i] ("ph"), T2[a,b,i,j] ("pphh"),
 * Gamma[G,p,q] with the No hole states first.  Complex tensors are
 * interleaved (re, im) doubles.
 */
#ifndef CC4S_CC_H
#define CC4S_CC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CC4S_OK 0
#define CC4S_ERR_INVALID_ARGUMENT 1
#define CC4S_ERR_BAD_SHAPE 2
#define CC4S_ERR_OUT_OF_MEMORY 3
#define CC4S_WARN_NOT_CONVERGED 4 /* warning: results are valid */
#define CC4S_ERR_DIIS_SINGULAR 5
#define CC4S_ERR_CUDA 6
#define CC4S_ERR_TIMEOUT 7
#define CC4S_ERR_STATE 8
#define CC4S_ERR_NON_FINITE 9
#define CC4S_ERR_UNSUPPORTED 10

#define CC4S_METHOD_CCSD 0
#define CC4S_METHOD_CCD 1
#define CC4S_METHOD_DRCCD 2

#define CC4S_PRECISION_FP64 0
#define CC4S_PRECISION_SPLIT2 2
#define CC4S_PRECISION_SPLIT3 3

#define CC4S_MIXER_DIIS 0
#define CC4S_MIXER_LINEAR 1

#define CC4S_MAX_HISTORY 256

typedef struct cc4s_cc_handle cc4s_cc_handle;

/* Options of the CoupledCluster step; defaults as in
 * src/main/algorithms/CoupledCluster.hpp:45-49 and the mixers. */
typedef struct {
  int method;                   /* "method" (default Ccsd), CoupledCluster.cxx:80 */
  int precision;                /* FP64 (default) or split-precision tensor-core form */
  int mixer;                    /* "mixer.type", CoupledCluster.cxx:96 */
  int max_residua;              /* "mixer.maxResidua" (4), DiisMixer.cxx:33 */
  double ratio;                 /* "mixer.ratio" (1.0), LinearMixer.cxx:32 */
  int max_iterations;           /* "maxIterations" (16) */
  double energy_convergence;    /* "energyConvergence" (1e-7) */
  double amplitudes_convergence;/* "amplitudesConvergence" (1e-6) */
  double level_shift;           /* "levelShift" (0) */
  int64_t integrals_slice_size; /* "integralsSliceSize" (0 = No), Ccsd.cxx:287-289 */
  int ppl;                      /* "ppl" (1), Ccsd.cxx:95 */
  int device;                   /* CUDA device ordinal */
  int profile;                  /* 1: time every contraction launch (CUDA events) */
  int linearized;               /* "linearized" (0), Drccd only, Drccd.cxx:53-55 */
  int adjacent_pairs_exchange;  /* "adjacentPairsExchange" (0), Drccd only, Drccd.cxx:56-58 */
  double precision_refinement;  /* split form only: once the residuum norm falls below this
                                   value the remaining iterations run in FP64, so the
                                   converged amplitudes solve the FP64 equations (0: off) */
} cc4s_cc_options;

typedef struct {
  double correlation, direct, exchange, second_order; /* energy.* outputs */
  double correlation_imag;     /* imaginary part of the complex energy */
  int iterations;              /* iterations performed */
  int converged;               /* convergenceReached */
  int history_len;
  double energy[CC4S_MAX_HISTORY];        /* per iteration: E */
  double delta_energy[CC4S_MAX_HISTORY];  /* dE */
  double residuum_norm[CC4S_MAX_HISTORY]; /* dR (DIIS-extrapolated change norm) */
  double seconds[CC4S_MAX_HISTORY];       /* device time of the iteration */
  double flops_per_iteration;  /* FP64-equivalent flops of one residual (this schedule) */
  int refined_from;            /* split form with precision_refinement: first iteration run
                                  in FP64 (1-based; 0: none) */
} cc4s_cc_result;

typedef struct {
  uint64_t gemm_launches;      /* tensor-core contraction kernels launched so far */
  uint64_t other_launches;     /* bandwidth kernels launched so far */
  uint64_t device_bytes;       /* device memory held by the handle */
  double flops_per_residual;   /* FP64-equivalent flops of one residual */
  /* with options.profile: contraction launches of the last residual */
  double gemm_seconds, gemm_flops;   /* all launches */
  double top_seconds, top_flops;     /* the most expensive launch */
  int gemm_profiled_launches;
  double split_seconds, split_flops;  /* the split-precision launches among them */
  int split_launches;
} cc4s_cc_stats;

/* Outcome of the Lambda solve behind cc4s_cc_relaxed_gradient. */
typedef struct {
  int iterations;           /* Jacobi + mixer iterations of the Lambda equations */
  int converged;            /* 1 if the norm of the last change fell below the threshold */
  double residuum_norm;     /* norm of the last (extrapolated) change of Lambda */
  double prepare_seconds;   /* recorded forward residual + energy gradients */
  double vjp_seconds;       /* one Lambda iteration (one transposed-Jacobian product) */
  double gradient_seconds;  /* final product with dR/dGamma and the integrals */
} cc4s_cc_lambda_result;

/* Fills the defaults of the reference. */
void cc4s_cc_default_options(cc4s_cc_options* opt);

/* Replaces the construction of CoupledCluster with its method and mixer
 * (CoupledCluster.cxx:79-103: CoupledClusterMethodFactory::create,
 * MixerFactory::create). */
int cc4s_cc_create(const cc4s_cc_options* opt, cc4s_cc_handle** h);

/* Replaces the inputs slicedEigenEnergies {h, p} and slicedCoulombVertex
 * (CoupledCluster.cxx:59-66, Ccsd.cxx:110-117).  gamma is Gamma[NG, Np, Np]
 * with Np = No + Nv, holes first (SliceOperator.cxx:95-131).  half_grid
 * selects the real integral path V = Re*Re + Im*Im
 * (VertexCoulombIntegrals.cxx:45-52); otherwise V_pqsr = sum conj(G_sp) G_qr.
 * The coulombIntegrals input is not needed: the integral slices are formed on
 * the device from gamma. */
int cc4s_cc_set_inputs(cc4s_cc_handle* h, const double* eps_h, int64_t No,
                       const double* eps_p, int64_t Nv, const double* gamma, int64_t NG,
                       int is_complex, int half_grid);

/* Replaces the "initialAmplitudes" input (CoupledCluster.cxx:70-75).
 * T1[a,i], T2[a,b,i,j] column-major; complex interleaved on the complex path. */
int cc4s_cc_set_initial_amplitudes(cc4s_cc_handle* h, const double* T1, const double* T2);

/* Replaces CoupledCluster::run<F,TE> (CoupledCluster.cxx:56-191): the iteration
 * loop, Jacobi update, mixer and energy.  Returns CC4S_WARN_NOT_CONVERGED when
 * maxIterations is reached (results are still filled in). */
int cc4s_cc_run(cc4s_cc_handle* h, cc4s_cc_result* out);

/* Replaces the "amplitudes" output (CoupledCluster.cxx:186-190). */
int cc4s_cc_get_amplitudes(cc4s_cc_handle* h, double* T1, double* T2);

/* One residual evaluation, Ccsd::getResiduum (Ccsd.cxx:77-378 / 382-633),
 * on caller amplitudes (T1 == T2 == NULL: first iteration).  Outputs R1[a,i],
 * R2[a,b,i,j] column-major. */
int cc4s_cc_residual(cc4s_cc_handle* h, const double* T1, const double* T2, double* R1,
                     double* R2);

/* Adjoint form, at the current (frozen) amplitudes — after cc4s_cc_run or
 * cc4s_cc_set_initial_amplitudes.  Replaces the transition structure factor of
 * FiniteSizeCorrection::calculateTransitionStructureFactor
 * (src/main/algorithms/FiniteSizeCorrection.cxx:50-133) with unit singular
 * vectors and Coulomb potential:
 *   S_of_G[G] = Re sum conj(Gamma_G,ai) Gamma_G,jb (2 Tt_abij - Tt_abji),
 *   Tt = T2 + T1 T1, which is dE_c/dV(G) when Gamma_G scales as sqrt(V(G)).
 * dE_dGamma (optional, real half-grid path only): the gradient of E_c with
 * respect to the caller's vertex Gamma[G,p,q] (same layout; complex input gives
 * d/dRe + i d/dIm), nonzero in the particle-hole block.  Either output may be NULL. */
int cc4s_cc_backward(cc4s_cc_handle* h, double* S_of_G, double* dE_dGamma);

/* Transposed-Jacobian product of the residual (Ccsd / Ccd, real half-grid and
 * complex paths): at amplitudes T1 [Nv,No], T2 [Nv,Nv,No,No] (reference layout,
 * as for cc4s_cc_residual) and an adjoint R1bar, R2bar of the residual (same layout),
 *   T1bar, T2bar = Rbar^T dR/dT   (T2bar projected on T_abij = T_baji),
 *   dGamma       = Rbar^T dR/dGamma in the caller's vertex layout (may be NULL).
 * Complex path: the real pairing Re sum conj(Rbar) R is differentiated, every
 * adjoint is d/dRe + i d/dIm.  The adjoint of Ccsd::getResiduum (Ccsd.cxx:77-378,
 * complex :382-633), built by replaying the recorded residual backwards. */
int cc4s_cc_residual_vjp(cc4s_cc_handle* h, const double* T1, const double* T2,
                         const double* R1bar, const double* R2bar, double* T1bar, double* T2bar,
                         double* dGamma);

/* Relaxed gradient of the converged correlation energy (after cc4s_cc_run, Ccsd /
 * Ccd, real half-grid and complex paths): solves the Lambda equations
 *   (dR/dT + D)^T lambda = -dE/dT
 * with the amplitude iteration's Jacobi update, level shift and mixer, each
 * iteration one transposed-Jacobian product, and returns
 *   dE_dGamma = dE_c/dGamma|_T + lambda^T dR/dGamma
 * in the caller's vertex layout (complex input: d/dRe + i d/dIm; on the complex
 * path the amplitude iteration keeps T_abij = T_baji, exact for a vertex with
 * Gamma_qp = conj(Gamma_pq), so directional derivatives are meaningful along
 * directions that keep that symmetry).  Converged when
 * the norm of the change of lambda is below `convergence`; otherwise status 4.
 * Replaces finite differences of CoupledCluster::run (CoupledCluster.cxx:56-191)
 * around converged amplitudes. */
int cc4s_cc_relaxed_gradient(cc4s_cc_handle* h, int max_iterations, double convergence,
                             double* dE_dGamma, cc4s_cc_lambda_result* out);

/* Options of the perturbative triples step. */
typedef struct {
  int64_t block_size;   /* virtual indices per block of the (a,b,c) loop (0: automatic,
                           the largest block whose (block * No)^3 array fits the L2 cache) */
  int formulation;      /* complex path: 0 = PerturbativeTriples (atrip, Equations.hpp
                           getEnergyDistinct: Re conj(W) Z), 1 = PerturbativeTriplesReference
                           (PerturbativeTriplesReference.cxx:136-173: Re conj(W) conj(Z));
                           the same on the real path; ignored when cT = 1 */
  int cT;               /* "cT" of PerturbativeTriplesReference (:70-71, :92-109, :178-179):
                           1 = completely renormalised triples, E = sum M Z with M built
                           from the intermediates of ct::getCompleteTriples
                           (CompleteTriples.cxx:11-118) in place of V_bcdk, V_jklc */
} cc4s_cc_triples_options;
typedef struct {
  double correlation;     /* energy.correlation of the step */
  double seconds;         /* device time of the block loop */
  double setup_seconds;   /* device time of the integral slices pphh, ppph, hhhp (and of
                             the cT intermediates) */
  double flops;           /* 2 No^3 Nv^3 (No + Nv), the reference's count
                             (PerturbativeTriples.cxx, atripDryRun) */
  double executed_flops;  /* flops of the contractions launched (whole block triples) */
  int64_t block_size;
  int64_t block_triples;  /* blocks A <= B <= C evaluated */
  double phase_seconds[4];  /* options.profile of the handle: device time of the singles,
                               particle contractions, hole contractions and energy kernel */
  double mp2_energy;      /* second-order energy of the handle's integrals in its basis,
                             sum Re(2 M_abij V_abij - M_abij V_abji), M = conj(V)/D
                             (PerturbativeTriplesStar.hpp:79-99): the denominator of the
                             (T*) ratio; starCorrection = (sum of the caller's CBS pair
                             energies) / mp2_energy * correlation */
  double cr_denominator;  /* cT = 1: the denominator of the CR-(T) energy that
                             PerturbativeTriplesReference prints (:187-195),
                             ct::getDenominator (CompleteTriples.cxx:120-165);
                             CR-(T) = correlation / cr_denominator.  0 when cT = 0 */
} cc4s_cc_triples_result;
void cc4s_cc_triples_default_options(cc4s_cc_triples_options* opt);
/* Perturbative triples energy at the current amplitudes (after cc4s_cc_run or
 * cc4s_cc_set_initial_amplitudes).  Replaces the steps
 *   - name: PerturbativeTriples           (src/main/algorithms/PerturbativeTriples.cxx:27-255,
 *                                           the atrip tuple loop)
 *   - name: PerturbativeTriplesReference  (src/main/algorithms/PerturbativeTriplesReference.cxx:56-222,
 *                                           cT = 0 or 1)
 *     in:  {amplitudes, coulombIntegrals, slicedEigenEnergies}
 *     out: {energy: {correlation, unit}}
 * The integral slices pphh, ppph and hhhp are formed on the device from the
 * vertex given to cc4s_cc_set_inputs; the contractions run in the handle's
 * precision (FP64 or the split form); on the complex path the hole integrals
 * enter conjugated as in both reference steps. */
int cc4s_cc_perturbative_triples(cc4s_cc_handle* h, const cc4s_cc_triples_options* opt,
                                 cc4s_cc_triples_result* out);
/* Options of the finite-size correction step. */
typedef struct {
  int interpolation_grid_size;  /* "interpolationGridSize" (20), FiniteSizeCorrection.cxx:143 */
  double unit_factor;           /* product of the reference's unit factors toCoulombVertexUnits *
                                   (grid unit / Gamma unit^2) = 1 / (grid unit^2 * potential
                                   unit); 1 for inputs in consistent units */
} cc4s_cc_fsc_options;
typedef struct {
  double correction, uncorrected, corrected;  /* energy.{correction, uncorrected, corrected} */
  double seconds;                             /* device time (uploads, S(G), interpolation) */
  int64_t box[3];                             /* lattice box of the interpolated S(G) */
} cc4s_cc_fsc_result;
void cc4s_cc_fsc_default_options(cc4s_cc_fsc_options* opt);
/* Finite-size correction at the current amplitudes.  Replaces the step
 *   - name: FiniteSizeCorrection  (src/main/algorithms/FiniteSizeCorrection.cxx:28-310)
 *     in:  {amplitudes, coulombVertexSingularVectors, slicedCoulombVertex, coulombPotential,
 *           gridVectors, interpolationGridSize}
 *     out: {transitionStructureFactor, energy: {correction, uncorrected, corrected, unit}}
 * singular_vectors: U[G,F] column-major complex interleaved (NGG x NG, NG the vertex
 * rows given to cc4s_cc_set_inputs; NULL: the identity, NGG = NG); coulomb_potential:
 * V[G] (NULL: 1); grid_vectors: [3, NGG] column-major (the cartesian G vectors);
 * reciprocal_basis: the rows Gi, Gj, Gk of the gridVectors metaData.  S_of_G
 * (optional, [NGG]) receives transitionStructureFactor.  The structure factor
 * (FiniteSizeCorrection.cxx:50-133) is formed on the device without the NGG vertex
 * rows; the Catmull-Rom tricubic interpolation over the (2N)^3 NGG refined points
 * runs on the device too (on one rank the reference counts every point). */
int cc4s_cc_finite_size_correction(cc4s_cc_handle* h, const double* singular_vectors,
                                   int64_t NGG, const double* coulomb_potential,
                                   const double* grid_vectors, const double* reciprocal_basis,
                                   const cc4s_cc_fsc_options* opt, double* S_of_G,
                                   cc4s_cc_fsc_result* out);
int cc4s_cc_get_stats(const cc4s_cc_handle* h, cc4s_cc_stats* out);

/* Correlation energy of amplitudes that already live in device memory, computed
 * without allocating any device memory.  No counterpart in the reference: this
 * is for callers that cannot allocate at the point of the call (hosts whose
 * device memory is entirely owned by their own pool, or loops that must not
 * pay for the device synchronisation a cudaFree implies).
 * Inputs (device pointers, reference column-major layout, complex interleaved
 * when is_complex): T1[a,i], T2[a,b,i,j] and V_abij (the "pphh" integrals).
 * Output: energy[0..3] (device) = direct, exchange, and their imaginary parts,
 * with correlation = direct + exchange as in CoupledCluster::getEnergy.
 * Temporary data lives in a fixed 2 MiB device array (nothing in it, nor in
 * energy, has to start at zero), so No <= 256
 * (larger systems are rejected with CC4S_ERR_BAD_SHAPE).  Each call made outside
 * stream capture looks up that array's device address (allocating nothing);
 * calls during capture reuse the last address found on the device, so make the
 * first call on a device before any stream capture (else CC4S_ERR_STATE).  A
 * CUDA error already pending from the caller's earlier work is reported as
 * CC4S_ERR_CUDA without launching and is left pending for the caller.  Every
 * call shares the array: calls whose kernels overlap on the GPU (different
 * streams, no ordering) race.  stream is a cudaStream_t (NULL: the legacy
 * default stream).  Errors: cc4s_cc_last_error(NULL). */
int cc4s_cc_energy_noalloc(const double* T1, const double* T2, const double* Vpphh, int64_t No,
                           int64_t Nv, int is_complex, double* energy, void* stream);

/* Releases the handle and its device memory. */
int cc4s_cc_destroy(cc4s_cc_handle* h);

/* Message of the last failure on this handle (or of the last failed create). */
const char* cc4s_cc_last_error(const cc4s_cc_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* CC4S_CC_H */
