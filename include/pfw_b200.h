/*
 * pfw_b200.h — C ABI of libpfw_b200.so, the B200 (sm_100a) force-evaluation
 * hot path of PotentialFrameWork.jl: cell-list neighbour construction,
 * SmoothPair / Lennard-Jones pair energy-force-virial, and ACE site
 * energy-force-virial.
 *
 * Conventions (identical to the reference's numeric boundary):
 *   - lengths in Å, energies in eV, forces in eV/Å;
 *   - positions X are 3×N column-major (X[3*i + a]), original atom order;
 *   - the cell H is 3×3 column-major with COLUMNS = cell vectors
 *     (H[a + 3*b] = component a of cell vector b), as AtomsBase.cell_vectors;
 *   - forces are returned 3×N column-major in original atom order;
 *   - the virial is 3×3 column-major, W = -Σ d ⊗ g over interactions;
 *   - species are integer channels 0..nz-1 (the caller maps ChemicalSpecies).
 *
 * Every entry point returns a pfw_status; the message of the last failure of a
 * workspace is available from pfw_last_error(ws).  No entry point traps or
 * asserts on the device.  One workspace per host thread (not reentrant), as
 * the reference's Workspace (PairPotentials/evaluation.jl:29).
 */
#ifndef PFW_B200_H
#define PFW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The Julia shim maps EINVAL → ArgumentError (storage.jl:89-93,134),
 * EDOMAIN → DomainError (NeighbourList/gpu.jl:395), ESHAPE → DimensionMismatch. */
typedef enum pfw_status {
  PFW_OK = 0,
  PFW_EINVAL = 1,     /* invalid argument: nonfinite/dependent cell, bad cutoff ... */
  PFW_EDOMAIN = 2,    /* coincident atoms with a singular model, nonfinite output */
  PFW_ESHAPE = 3,     /* array shape mismatch */
  PFW_ECAPACITY = 4,  /* internal capacity overflow (retried internally) */
  PFW_ECUDA = 5,      /* CUDA runtime error */
  PFW_ETIMEDOUT = 6,  /* a bounded device wait ran out */
  PFW_ESTATE = 7      /* call order error: no geometry / no model loaded */
} pfw_status;

/* request bits, mirroring AtomsCalculators Energy()/Forces()/Virial()
 * (NeighbourList/execution.jl:4-12 normalize_properties). */
#define PFW_REQ_ENERGY 1u
#define PFW_REQ_FORCES 2u
#define PFW_REQ_VIRIAL 4u

/* arithmetic forms */
#define PFW_PRECISION_FP64 0   /* plain path: every operation in FP64 */
#define PFW_PRECISION_MIXED 1  /* FP32 pair/ACE arithmetic, FP64 wrap + Kahan FP64 E/W */

typedef struct pfw_options {
  int32_t precision;            /* PFW_PRECISION_FP64 or PFW_PRECISION_MIXED */
  int32_t bruteforce_threshold; /* Workspace(bruteforce_threshold=32) (storage.jl:59-65) */
  int32_t device;               /* CUDA device ordinal */
  int32_t reserved;
} pfw_options;

typedef struct pfw_ws pfw_ws;

/* ---- lifecycle -------------------------------------------------------- */
/* Library version string "major.minor.patch". */
const char* pfw_version(void);

/* Replaces NeighbourList.Workspace(; width, precision, bruteforce_threshold)
 * (NeighbourList/storage.jl:59-65).  opts may be NULL for defaults
 * (FP64, threshold 32, device 0). */
pfw_status pfw_ws_create(const pfw_options* opts, pfw_ws** out);
void pfw_ws_destroy(pfw_ws* ws);
/* Message of the last failed call on this workspace ("" if none). */
const char* pfw_last_error(const pfw_ws* ws);

/* ---- geometry --------------------------------------------------------- */
/* Host-side geometry upload; replaces the extraction half of prepare!
 * (storage.jl:130-180).  X: 3×n, H: 9, pbc: 3 flags, species: n channels. */
pfw_status pfw_set_geometry(pfw_ws* ws, int64_t n, const double* X, const double* H,
                            const uint8_t pbc[3], const int32_t* species);
/* Same, but X and species are DEVICE pointers already resident in HBM
 * (no host↔device copy); H and pbc are host arrays. */
pfw_status pfw_set_geometry_device(pfw_ws* ws, int64_t n, const double* X_dev,
                                   const double* H, const uint8_t pbc[3],
                                   const int32_t* species_dev);

/* Domain decomposition (no counterpart in the single-process reference,
 * README.md:327): atoms [0, n_owned) of the current single-system geometry
 * are this rank's own, the rest are ghost copies of other ranks' atoms.
 * Forces are computed for every atom (exact for owned atoms whose
 * neighbourhood the ghosts cover), but energy and virial count only the
 * owned atoms' shares — half of every directed pair of an owned centre, the
 * site terms of owned sites — so the ranks' energies and virials sum to the
 * whole system's.  -1 (the default after every geometry upload) = all. */
pfw_status pfw_set_owned(pfw_ws* ws, int64_t n_owned);

/* Slab decomposition, the per-step exchange's device half (no counterpart in
 * the reference): of a rank's n owned atoms (X_dev 3×N, species_dev on the
 * device), the ones whose fractional coordinate along the slab axis,
 * f = frac_row·x (frac_row: that row of H⁻¹), lies below lo + d (lower band)
 * and at or above hi - d (upper band), in their owned order, written as
 * (x, y, z, species) quadruples of doubles with shift_lower / shift_upper
 * (Cartesian, Å) added: the neighbouring ranks' ghost atoms.  lower_dev and
 * upper_dev hold 4·n doubles; counts_dev[0..1] receive the band sizes.  Runs
 * on the workspace's stream without synchronising. */
pfw_status pfw_slab_bands(pfw_ws* ws, int64_t n, const double* X_dev, const int32_t* species_dev,
                          const double frac_row[3], double lo, double hi, double d, const double shift_lower[3],
                          const double shift_upper[3], double* lower_dev, double* upper_dev, int32_t* counts_dev);

/* ---- pair models ------------------------------------------------------ */
/* SmoothPair(labels, amplitudes, cutoff): U_ab(r) = A_ab (1 - r²/c²)³
 * (PairPotentials/models.jl:28-44 and PreparedSmooth :138-176).
 * A is nz×nz symmetric, indexed by species channel. */
pfw_status pfw_pair_model_smooth(pfw_ws* ws, int32_t nz, const double* A, double cutoff);
/* lennard_jones(; epsilon, sigma, radius): energy-shifted LJ
 * (PairPotentials/lennard_jones.jl:5-33). */
pfw_status pfw_pair_model_lj(pfw_ws* ws, double epsilon, double sigma, double cutoff);

/* Verlet skin reuse of the pair list, the reference's GPU skin path
 * (gpu_skin!, gpu_displacements!, NeighbourList/gpu.jl:404-549): with
 * skin > 0 (Å) the pair evaluation of a single system builds the directed
 * snapshot within cutoff + skin once and reuses it while the atom count, cell
 * and periodicity are unchanged and no atom moved more than skin/2 (original
 * coordinates) since the build; 0 (the default) rebuilds on every call, as
 * evaluate! does.  FP64 workspaces only.  Pairs within about one ulp of the
 * cutoff may be selected differently from a rebuild (the displacement is
 * X_j - X_i + H·S from the original coordinates). */
pfw_status pfw_pair_set_skin(pfw_ws* ws, double skin);
/* List builds and reuses since the workspace was created. */
pfw_status pfw_pair_skin_stats(pfw_ws* ws, int64_t* builds, int64_t* reuses);

/* ---- ACE models ------------------------------------------------------- */
/* Packed resolved-ACE tables; the host builds them from the resolved TOML v1
 * schema (ACE/resolved.jl:103-142), mirroring pack_model (ACE/adaptation.jl:78-98).
 * All indices are 0-based.  Ragged spline tables are padded to the longest
 * node list of the family.  Only the default basis policy is packed: the
 * invariant mask is applied to WB by the host; pair/reference flags per species. */
typedef struct pfw_radial_family {
  int32_t nchannels;            /* radial functions per species pair (nR or nQ) */
  int32_t nknots;               /* max number of spline nodes (intervals = nknots-1) */
  const int32_t* lengths;       /* [nz*nz] number of nodes of pair (iz,jz) at iz*nz+jz */
  const double* nodes;          /* [nz*nz][nknots] */
  const double* coeff;          /* [nz*nz][nknots-1][nchannels][4] power 0..3 */
  const double* transform;      /* [nz*nz][6] a, rin, r0, yin, ycut, rcut */
  const int32_t* powers;        /* [nz*nz][2] p, q */
  const int32_t* envelope_kind; /* [nz*nz] 1 PolyEnvelope2sX, 2 ACE1_PolyEnvelope1sR, 3 PolyEnvelope1sR */
  const double* envelope;       /* [nz*nz][5] parameters in resolved.jl:73-78 order */
} pfw_radial_family;

typedef struct pfw_ace_tables {
  int32_t nz;                   /* species channels, 1..16 */
  int32_t lmax;                 /* harmonics degree (L2, l*l+l+m order), 0..6 */
  pfw_radial_family radial;     /* R channels */
  pfw_radial_family pair;       /* Q (pair) channels */
  int32_t ndensity;             /* D, at most 65534 */
  const int32_t* density;       /* [D][2] (radial channel, harmonic index) */
  int32_t nproducts;            /* P, at most 65535 */
  const int32_t* product_offsets; /* [P+1] CSR into product_factors */
  const int32_t* product_factors; /* density indices of each product: 1 to 4 per
                                     product (correlation order <= 4; longer or empty
                                     products are rejected with PFW_EINVAL) */
  int32_t nbasis;               /* nB invariants (rows of the coupling) */
  int32_t ncoupling;            /* stored coupling entries */
  const int32_t* coupling_rows; /* [nnz] invariant index, column-major (CSC) order */
  const int32_t* coupling_cols; /* [nnz] product index */
  const double* coupling_vals;  /* [nnz] */
  const double* WB;             /* [nz][nbasis] readout, mask applied */
  const double* Wpair;          /* [nz][nQ] */
  const double* reference;      /* [nz] reference energies (0 when disabled) */
  const uint8_t* pair_allowed;  /* [nz] pair term enabled for neighbour species */
  double cutoff;                /* search cutoff = max rcut over channels (cpu.jl:316) */
  int32_t angular_kind;         /* 0 real spherical Y_lm, 1 real solid r^l·Y_lm (BlockAngular
                                   solid=true, ACE/angular_blocks.jl:25-48; the May30 models) */
} pfw_ace_tables;

/* Load an ACE model (copies every table to the device). */
pfw_status pfw_ace_model_load(pfw_ws* ws, const pfw_ace_tables* tables);

/* Schedule of the ACE site kernel: edges per chunk (8 or 16) and site
 * groups of 64 threads per CTA (1..8); 0, 0 = automatic (largest working set
 * that fits).  The autotuner (pfw_b200/autotune.py) times the candidates on
 * the caller's workload and caches the choice.  Returns PFW_EINVAL when the
 * schedule does not fit the model in shared memory. */
pfw_status pfw_ace_set_schedule(pfw_ws* ws, int32_t chunk, int32_t groups);

/* ---- evaluation ------------------------------------------------------- */
/* Replaces evaluate!(w, sys, p; request) (PairPotentials/evaluation.jl:31-52)
 * for the loaded pair model, or AC.energy_forces_virial(sys, ACECalculator)
 * (ACE/calculators.jl:48-96) when model == PFW_MODEL_ACE.  Host outputs; any may
 * be NULL when not requested.  E: 1, F: 3×n original order, W: 9. */
#define PFW_MODEL_PAIR 0
#define PFW_MODEL_ACE 1
pfw_status pfw_evaluate(pfw_ws* ws, int32_t model, uint32_t request,
                        double* E, double* F, double* W);
/* Same with DEVICE outputs (E: 1 double, F: 3n, W: 9) — no host copies, no sync. */
pfw_status pfw_evaluate_device(pfw_ws* ws, int32_t model, uint32_t request,
                               double* E_dev, double* F_dev, double* W_dev);
/* Per-site energies of the last ACE evaluation (original order, host). */
pfw_status pfw_site_energies(pfw_ws* ws, double* energies);
/* Number of in-cutoff unordered pairs of the last pair evaluation's geometry. */
pfw_status pfw_last_pair_count(pfw_ws* ws, int64_t* npairs);

/* ---- neighbour snapshot ------------------------------------------------ */
/* neighbour_list(sys, cutoff) + neighbours(list, i) (NeighbourList/interface.jl:47-151).
 * Two calls: count builds the directed snapshot on the device and returns the
 * number of directed entries M; fill copies it out in original order:
 * offsets [n+1], j [M] (0-based original index), S [3M] (integer shifts),
 * R [3M] (Å, R = X[j] - X[i] + H·S up to rounding).  Any output may be NULL. */
pfw_status pfw_neighbour_count(pfw_ws* ws, double cutoff, int64_t* total);
pfw_status pfw_neighbour_fill(pfw_ws* ws, int64_t* offsets, int32_t* j, int32_t* S, double* R);

/* ---- batches of independent systems ------------------------------------ */
/* Replaces a loop of evaluate! / energy_forces_virial calls over independent
 * structures, such as the training set of design_matrix (ACE/fitting.jl:18-67),
 * with one launch over all of them.  nsys systems; their atoms are
 * concatenated system after system: system s owns atoms
 * [atom_offsets[s], atom_offsets[s+1]) (atom_offsets[0] = 0, nsys+1 entries).
 * H holds 9 doubles per system (column-major, columns = cell vectors), pbc 3
 * flags per system.  X (3×N) and species (N) are host arrays for
 * pfw_set_batch and device arrays for pfw_set_batch_device; offsets, H and
 * pbc are always host arrays.  Replaces the single-system geometry. */
pfw_status pfw_set_batch(pfw_ws* ws, int32_t nsys, const int64_t* atom_offsets, const double* X,
                         const double* H, const uint8_t* pbc, const int32_t* species);
pfw_status pfw_set_batch_device(pfw_ws* ws, int32_t nsys, const int64_t* atom_offsets, const double* X_dev,
                                const double* H, const uint8_t* pbc, const int32_t* species_dev);
/* New positions (3×N, same systems, cells and species) for the next
 * evaluation; on_device != 0: X is device memory (queued, no sync).  A
 * captured batch graph stays valid. */
pfw_status pfw_batch_update_positions(pfw_ws* ws, const double* X, int32_t on_device);
/* Dense energy/force/virial design rows of the loaded ACE model for the
 * current geometry or batch: replaces design_matrix(X, model, ps, env, H;
 * fit_pair=true) (ACE/fitting.jl:18-67) for every structure at once, the
 * assembly ACEfit stacks.  Rows of system s start at 10·s + 3·(atoms before
 * s): the energy row, 3 force rows per atom (original order, component
 * fastest), the 9 virial rows (column-major 3×3); columns (row-major, leading
 * dimension ld ≥ cols) are vec(WB) (species block z at z·nbasis + b) then
 * vec(Wpair) (nz·nbasis + z·nQ + q), so A·[vec(WB); vec(Wpair)] + baseline
 * reproduces [E; F; W].  baseline[s] (optional, nsys) is the structure's sum
 * of reference energies (the energy row's baseline; the other rows' are 0).
 * Rows are deterministic.  PFW_ESHAPE when the buffer is too small. */
pfw_status pfw_ace_design_shape(pfw_ws* ws, int64_t* rows, int64_t* cols);
pfw_status pfw_ace_design_matrix(pfw_ws* ws, double* A, int64_t ld, int64_t rows_capacity, double* baseline);
pfw_status pfw_ace_design_matrix_device(pfw_ws* ws, double* A_dev, int64_t ld, int64_t rows_capacity,
                                        double* baseline_dev);

/* Per-structure fitting features of the loaded ACE model: nz·(nB + nQ)
 * values per system, laid out [Σ_i B_i of species block z (nB each, z =
 * 0..nz-1), then Σ_{i,j} Q[j,:] of species block z (nQ each)] — the energy
 * row of design_matrix (ACE/fitting.jl:28-29) without the reference
 * energies. */
pfw_status pfw_ace_feature_count(pfw_ws* ws, int32_t* nfeat);
/* Batch evaluation.  E: nsys, F: 3×N (original order), W: 9 per system,
 * features: nfeat per system (ACE only; NULL skips them).  Any output may be
 * NULL when not requested.  Host outputs, synchronous. */
pfw_status pfw_evaluate_batch(pfw_ws* ws, int32_t model, uint32_t request, double* E, double* F,
                              double* W, double* features);
/* Same with DEVICE outputs; still checks device status before returning. */
pfw_status pfw_evaluate_batch_device(pfw_ws* ws, int32_t model, uint32_t request, double* E_dev,
                                     double* F_dev, double* W_dev, double* features_dev);
/* ACE batch through a CUDA graph: the first call (and any call after the
 * batch, model, schedule, request or output pointers changed) evaluates
 * eagerly to plan, sizes the environment buffers with 25 % headroom and
 * captures cell lists + environments + site kernel + force gather + per-system
 * outputs as one graph on the workspace stream; every call then launches the
 * graph and returns without synchronising.  Requires fully periodic systems.
 * pfw_batch_graph_sync waits and reports device status: PFW_ECAPACITY when
 * moved positions outgrew the headroom (call again: it re-plans). */
pfw_status pfw_batch_graph_launch(pfw_ws* ws, uint32_t request, double* E_dev, double* F_dev,
                                  double* W_dev, double* features_dev);
pfw_status pfw_batch_graph_sync(pfw_ws* ws);

/* ---- learned per-atom surrogate ----------------------------------------- */
/* No GPU counterpart in the reference; the nearest CPU analogue is the
 * invariant head ACEFeatureEnergy (ACE/feature_energy.jl:1-86).  A FEATURE
 * MODEL (packed ACE tables restricted to low-order invariants: its nbasis
 * invariants B = C·P, then its pair channels Q, nin = nbasis + nQ features
 * per site) feeds an ensemble of MLPs per centre species,
 * nin → hidden → hidden → 1 with SiLU, BF16 weights and FP32 arithmetic.
 * Site energy = reference[z] + y_mean[z] + y_std[z]·mean over members;
 * forces and virial follow from dE/dfeature through the ACE pullback.  A site
 * falls back to the full ACE model (pfw_ace_model_load) when a standardised
 * feature leaves [x_lo, x_hi] or the ensemble standard deviation of its
 * energy exceeds tau (eV). */
typedef struct pfw_mlp_params {
  int32_t nz, members, nin, hidden;  /* members 1..4; nin, hidden multiples of 8 */
  const uint16_t* W1;   /* [nz][members][hidden][nin]    BF16 bit patterns */
  const float* b1;      /* [nz][members][hidden] */
  const uint16_t* W2;   /* [nz][members][hidden][hidden] BF16 (row = output) */
  const float* b2;      /* [nz][members][hidden] */
  const uint16_t* w3;   /* [nz][members][hidden]         BF16 */
  const float* b3;      /* [nz][members] */
  const double* x_mean; /* [nz][nin] feature standardisation */
  const double* x_std;
  const float* x_lo;    /* [nz][nin] accepted standardised range, margin included */
  const float* x_hi;
  const double* y_mean; /* [nz] standardisation of (site energy - reference) */
  const double* y_std;
  double tau;           /* gate on the ensemble standard deviation (eV) */
} pfw_mlp_params;

#define PFW_MODEL_SURROGATE 2

/* Load the feature model and (optionally, NULL) the MLP ensemble. */
pfw_status pfw_surrogate_load(pfw_ws* ws, const pfw_ace_tables* features, const pfw_mlp_params* mlp);
/* Per-site features of the current geometry (host, n × nin, original
 * order): the training inputs. */
pfw_status pfw_surrogate_features(pfw_ws* ws, double* features);
/* Sites of the last surrogate evaluation and how many fell back to ACE. */
pfw_status pfw_surrogate_stats(pfw_ws* ws, int64_t* fallback_sites, int64_t* sites);

/* Ensemble training with hand-written forward/backward kernels: mean squared
 * error on standardised site energies, Adam, one parameter vector per
 * (species, member): [W1 hidden×nin | b1 | W2 hidden×hidden | b2 | w3 | b3]
 * in FP32, nparams = hidden·nin + hidden² + 3·hidden + 1. */
typedef struct pfw_mlp_shape {
  int32_t nz, members, nin, hidden;
} pfw_mlp_shape;
typedef struct pfw_mlp_train_options {
  int32_t epochs, batch;   /* batch: samples per member per step (multiple of 32) */
  float lr, lr_final;      /* cosine decay from lr to lr_final */
  uint64_t seed;           /* per-member sample orders */
} pfw_mlp_train_options;
/* Gradient of the mean squared error over the samples of each species for
 * every (species, member) model: loss [nz·members], grad like params. */
pfw_status pfw_mlp_param_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params, int64_t n,
                              const float* X, const float* y, const int32_t* species, double* loss,
                              float* grad);
/* params: initial values in, trained values out.  X: n × nin standardised
 * features, y: n standardised targets, species: n channels (host arrays).
 * epoch_loss [epochs] (may be NULL): mean training loss over the models. */
pfw_status pfw_mlp_train(pfw_ws* ws, const pfw_mlp_shape* shape, float* params, int64_t n, const float* X,
                         const float* y, const int32_t* species, const pfw_mlp_train_options* options,
                         float* epoch_loss);

/* Energy + force training (feature_energy.jl:1-86 is the reference's CPU
 * analogue of the head; the force term has no counterpart there).  One
 * full-batch step over n samples on DEVICE buffers: X n × nin standardised
 * features, y n standardised energy targets, V [members][n][nin] the force
 * error of each member pulled back into standardised feature space (the
 * change of each site's features along ΔF; NULL: energy only), c [n] the
 * force weight of each sample; species is a HOST array.  The loss gradient
 * is wE·(energy MSE gradient) + Σ c·∂/∂θ(V·∇_x y) per (species, member)
 * model.  With grad_dev NULL it applies an Adam step (learning rate lr, step
 * number >= 1, moments m1/m2 like params); else it writes the gradient there
 * and leaves the parameters alone.  loss [nz·members] (host, may be NULL):
 * the energy MSE per model before the step. */
pfw_status pfw_mlp_ef_step(pfw_ws* ws, const pfw_mlp_shape* shape, float* params_dev, float* m1_dev, float* m2_dev,
                           int64_t n, const float* X_dev, const float* y_dev, const int32_t* species,
                           const float* V_dev, const float* c_dev, float wE, float lr, int64_t step, float* grad_dev,
                           double* loss);
/* ∂y/∂x (standardised) of every member at every sample: G_dev [members][n][nin]
 * (device), species a host array. */
pfw_status pfw_mlp_input_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params_dev, int64_t n,
                              const float* X_dev, const int32_t* species, float* G_dev);
/* Forces F_dev (3×n, original order, device) of the per-site feature
 * gradient field dEdx_dev (n × nin dE_i/dfeature_i, original order, device)
 * through the loaded surrogate feature model on the current geometry:
 * F_k = -Σ_i dEdx_i·∂feature_i/∂r_k (the surrogate's pullback pass). */
pfw_status pfw_surrogate_pullback(pfw_ws* ws, const double* dEdx_dev, double* F_dev);

/* ---- device peak probe ------------------------------------------------- */
/* Measured FP64 FMA throughput of the current device (TFLOP/s), used as the
 * FP64-pipe roofline denominator. */
pfw_status pfw_probe_fp64_peak(pfw_ws* ws, double* tflops);

/* Number of kernels this workspace has launched (monotone counter). */
uint64_t pfw_launch_count(const pfw_ws* ws);

/* Run the workspace's work on the caller's CUDA stream (a cudaStream_t; NULL
 * restores the workspace's own stream).  The caller keeps ownership. */
pfw_status pfw_set_stream(pfw_ws* ws, void* stream);

/* Stage diagnostics (the reference's gpu_stage_stamp!, ACE/gpu.jl:565-570):
 * when on, CUDA events bracket each stage of pfw_evaluate*; pfw_stage_times
 * waits for the last evaluation and returns its stage durations in ms:
 * [0] geometry (wrap, bins, sort), [1] main kernel (pair or ACE sites),
 * [2] reductions and force assembly, [3] neighbour-list build (ACE).
 * Returns the number of stages written (<= cap). */
pfw_status pfw_set_diagnostics(pfw_ws* ws, int32_t on);
int32_t pfw_stage_times(pfw_ws* ws, double* ms, int32_t cap);

/* ---- evaluation without any allocation ---------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts whose runtime owns every byte of device memory through its own pool,
 * and code that must not trigger the device-wide synchronisation a fresh
 * allocation can cause.  Evaluates SmoothPair (kind 0, params = nz×nz
 * amplitudes, finite and symmetric) or Lennard-Jones (kind 1, params =
 * {epsilon, sigma}) energy, forces and virial of one small system, brute
 * force, with the reference's minimum-image geometry.  Limits: n <=
 * PFW_NOALLOC_MAX_ATOMS atoms, an orthorhombic cell whose periodic lengths
 * exceed 2·cutoff (open axes allowed).  X_dev (3×n), species_dev (n) and the
 * outputs E_dev (1), F_dev (3×n, original order; required when forces are
 * requested) and W_dev (9) are DEVICE memory owned by the caller; H, pbc and
 * params are host arrays.  Work is queued on `stream` (a cudaStream_t, NULL =
 * default stream) without synchronising, so errors that depend on the data
 * arrive through status_dev (optional device int32, written when the queued
 * work completes): PFW_OK; PFW_EINVAL for a species channel outside [0, nz)
 * (SmoothPair) or negative, or a non-finite position; PFW_EDOMAIN for a
 * non-finite energy or virial (coincident atoms with Lennard-Jones).  The
 * outputs are undefined unless it reads PFW_OK.  The only scratch is a fixed
 * static device array of 64 blocks × 8 doubles plus one status word (4 KiB)
 * that every GPU loading the library keeps until exit; every call looks up
 * its device address (the first call on a device also loads the module, so
 * make that first call before any stream capture).  Calls that overlap on the
 * GPU share that array and race: serialise them.  The caller's current
 * device is left as it was.  A message is copied to errbuf (errlen bytes)
 * when an argument is rejected. */
#define PFW_NOALLOC_MAX_ATOMS 8192
pfw_status pfw_pair_evaluate_noalloc(int32_t device, void* stream, int64_t n, const double* X_dev,
                                     const int32_t* species_dev, const double H[9], const uint8_t pbc[3],
                                     int32_t kind, int32_t nz, const double* params, double cutoff,
                                     uint32_t request, double* E_dev, double* F_dev, double* W_dev,
                                     int32_t* status_dev, char* errbuf, int32_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* PFW_B200_H */
