/* aed.h -- C ABI of the B200 exact-diagonalisation engine (libaed.so).
 *
 * The engine replaces the hot path of ALPS `sparsediag`: the Sz-sector basis,
 * the Hamiltonian apply y = H*x and the ietl Lanczos iteration, for the spin-1/2
 * "spin" model on one GPU.  Every function returns an int status (AED_OK = 0,
 * negative on error); aed_last_error() describes the most recent failure on the
 * calling thread.  Vectors are plain device pointers to D elements of the
 * handle's precision (double for AED_FP64, float for AED_FP32).  All calls on a
 * handle are ordered on that handle's CUDA stream; calls that return host
 * scalars synchronise that stream.  One handle per host thread at a time.
 *
 * Reference paths are relative to the ALPS source tree.
 */
#ifndef AED_H
#define AED_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define AED_OK 0
#define AED_ERR_INVALID (-1)        /* bad argument / unsupported model        */
#define AED_ERR_NOMEM (-2)          /* device or host allocation failed        */
#define AED_ERR_ADMISSION (-3)      /* request refused: HBM budget exceeded    */
#define AED_ERR_CUDA (-4)           /* CUDA runtime error                      */
#define AED_ERR_TIMEOUT (-5)        /* bounded device wait gave up             */
#define AED_ERR_NOT_CONVERGED (-6)  /* MAX_ITERATIONS reached (iteration.h:80) */
#define AED_ERR_TRIDIAG (-7)        /* tridiagonal solver failed (tmatrix.h:144-145) */
#define AED_ERR_MISMATCH (-8)       /* replayed alpha/beta differ (lanczos.h:249-250,267-268) */
#define AED_ERR_CANCELLED (-9)      /* request cancelled before completion     */
#define AED_PENDING 1               /* aed_poll: request not finished yet      */

/* vector precision of a handle */
#define AED_FP64 0
#define AED_FP32 1

/* ---- model description ---------------------------------------------------
 * Replaces the model/lattice surface that hamiltonian_matrix reads
 * (src/alps/model/hamiltonian_matrix.hpp:224-231, 387-397): N spin-1/2 sites,
 * the Sz_total constraint (CONSERVED_QUANTUMNUMBERS="Sz") and the bond list in
 * graph order with per-bond couplings of the "spin" HAMILTONIAN
 * (lib/xml/models.xml.in:342-373):
 *   H = sum_s [-h_s Sz_s + D_s Sz_s^2]
 *     + sum_b [Jz_b Sz_i Sz_j + Jxy_b (S+_i S-_j + S-_i S+_j)/2 + K_b (S_i.S_j)^2]
 * All arrays are host memory and are copied by aed_create. */
typedef struct {
  int32_t n_sites;        /* N, 2..32                                          */
  int32_t n_up;           /* number of up spins: Sz_total = n_up - N/2          */
  int32_t n_bonds;        /* 0..AED_MAX_BONDS                                   */
  const int32_t* bond_s1; /* source site of each bond                           */
  const int32_t* bond_s2; /* target site of each bond (!= source)               */
  const double* bond_jz;  /* Jz of each bond                                    */
  const double* bond_jxy; /* Jxy of each bond                                   */
  const double* bond_k;   /* biquadratic K of each bond, or NULL for 0          */
  const double* site_h;   /* longitudinal field h per site, or NULL for 0       */
  const double* site_d;   /* single-ion D per site, or NULL for 0               */
} aed_model_desc;

#define AED_MAX_BONDS 128

/* Parameters read from an ALPS parameter file (the subset of the sparsediag
 * surface this engine supports; see aed_parse_parameters). */
typedef struct {
  int32_t n_sites;
  int32_t n_up;
  int32_t n_bonds;
  int32_t number_eigenvalues; /* NUMBER_EIGENVALUES, default 1 (sparsediag.h:110)        */
  int32_t max_iterations;     /* MAX_ITERATIONS, 0 = default min(10 D, 1000) (sparsediag.h:109) */
  int32_t has_site_terms;     /* h or D present                                         */
  int32_t two_s;              /* 2 local_S (1 .. 4); n_up is then the digit sum Sz_total + N S */
} aed_param_info;

/* Parse an ALPS parameter file ("KEY = value" lines, ';' or newline separated,
 * quoted strings, simple numeric expressions) into a bond list in ALPS graph
 * order.  Supported: MODEL="spin", local_S=1/2, LATTICE in {chain lattice,
 * open chain lattice, nnn chain lattice, nnn open chain lattice, square
 * lattice, open square lattice, anisotropic square lattice, ladder, open
 * ladder} with L/W, local_S in {1/2, 1, 3/2, 2} (info->two_s; aed_create_spin
 * for local_S > 1/2), couplings J, J0, J1, J', Jz, Jxy, Jz<n>, Jxy<n>, J<n>, K<n>,
 * h, D with the model library's defaults, CONSERVED_QUANTUMNUMBERS containing Sz, Sz_total,
 * NUMBER_EIGENVALUES, MAX_ITERATIONS.  TRANSLATION_SYMMETRY and TOTAL_MOMENTUM
 * select momentum sectors (aed_lattice_momenta); the bond list is the same.
 * Replaces the parameter path of SparseDiagFactory/DiagMatrix
 * (applications/diag/sparsediag/factory.C:17-30, applications/diag/diag.h:85-175,
 * src/alps/lattice/latticegraph.h:98-136, lib/xml/lattices.xml.in).
 * Call once with NULL arrays to get info->n_bonds, then with arrays of at least
 * that many entries (site arrays: n_sites entries). */
int aed_parse_parameters(const char* text, aed_param_info* info, int32_t* bond_s1, int32_t* bond_s2,
                         double* bond_jz, double* bond_jxy, double* bond_k, double* site_h,
                         double* site_d, int32_t bond_capacity, int32_t site_capacity);
/* The same for a graph of a lattice library (<GRAPH>: VERTEX id / type, EDGE
 * source / target / type; read_graph_xml, src/alps/lattice/graph.h:121-222,
 * chosen by LATTICE or GRAPH, graph_helper.h:653-684): the parameter text
 * gives the model and sector (its LATTICE is not read); n_vertices vertices
 * numbered from 0 with their types (NULL: all 0), n_edges edges in file order
 * with their types (NULL: all 0).  Bond b = edge b, with the couplings of its
 * edge type (Jz#, Jxy#, J#, K#); the site terms of a vertex are those of its
 * type (h#, D#, defaults h, D; models.xml.in:360-371). */
int aed_parse_graph_parameters(const char* text, int32_t n_vertices, const int32_t* vertex_type, int32_t n_edges,
                               const int32_t* edge_source, const int32_t* edge_target, const int32_t* edge_type,
                               aed_param_info* info, int32_t* s1, int32_t* s2, double* jz, double* jxy, double* kq,
                               double* site_h, double* site_d, int32_t bond_capacity, int32_t site_capacity);

/* ---- handles -------------------------------------------------------------- */
typedef struct aed_handle aed_handle;

/* Build the sector basis tables and the coupling tables on `device`.
 * Replaces hamiltonian_matrix::build_basis + build
 * (src/alps/model/hamiltonian_matrix.hpp:402-450; basis_states::build,
 * src/alps/model/basisstates.h:175-278).  No explicit matrix is stored: the
 * apply is matrix-free. */
int aed_create(const aed_model_desc* model, int precision, int device, aed_handle** out);
/* Device and pinned host memory of a destroyed handle goes back to a
 * per-process cache that the next aed_create reuses (no cudaMalloc / cudaFree
 * per handle in a create / solve / destroy loop). */
int aed_destroy(aed_handle* h);
/* Return the cached memory that no handle uses to the driver (device memory of
 * `device`, all cached pinned host memory).  No reference counterpart: the
 * reference's matrices are freed with their task. */
int aed_empty_cache(int device);
/* Allocate now the FP32 Lanczos basis store of a mixed-precision (AED_FP32)
 * spin-1/2 Sz-sector handle for `vectors` vectors, and the workspace of its
 * Rayleigh-Ritz step for the most Ritz vectors that step takes; both
 * otherwise grow inside the solves that need them, and are kept until
 * aed_destroy.  A long-running caller sizes it once so that no solve pays for
 * a device allocation.  No reference counterpart: the reference keeps no basis. */
int aed_reserve_basis(aed_handle* h, int32_t vectors);

/* ---- measurements ------------------------------------------------------- */
#define AED_OBS_SZ 0   /* <Sz_i>                       */
#define AED_OBS_SZSZ 1 /* <Sz_i Sz_j>                  */
#define AED_OBS_SPSM 2 /* <S+_i S-_j> (real vectors)   */
/* Expectation values <psi| O |psi> of site operators in a device vector of
 * the handle (not normalised by |psi|): out[p] for the site pair
 * (site_i[p], site_j[p]) (site_j ignored for AED_OBS_SZ).  The quantities
 * DiagMatrix::perform_measurements evaluates for MEASURE_AVERAGE, _LOCAL,
 * _CORRELATIONS and _STRUCTURE_FACTOR (applications/diag/diag.h:191-314 via
 * calculate(), :316-339), for the spin operators Sz, Splus, Sminus of the
 * handle's local spin (spin-1/2 handles of aed_create, spin-S handles of
 * aed_create_spin; models.xml.in:24-36).  Sz sectors only (momentum
 * sectors: aed_momentum_expectation). */
int aed_expectation(aed_handle* h, const void* psi, int32_t kind, int32_t n, const int32_t* site_i,
                    const int32_t* site_j, double* out);
/* Momentum sectors: <psi| sum_p O(site_i[p], site_j[p]) |psi> (the real part)
 * for a list of pairs whose sum is translation invariant, such as all pairs
 * of one distance class; *out gets the sum.  What perform_measurements
 * accumulates over the pairs of a distance class in a translation-invariant
 * sector (applications/diag/diag.h:236-258) before dividing by the class's
 * multiplicity, and over all pairs for the structure factor (:262-307).
 * Spin-1/2 and spin-S momentum sectors (aed_create_momentum,
 * aed_create_spin_momentum). */
int aed_momentum_expectation(aed_handle* h, const void* psi, int32_t kind, int32_t n, const int32_t* site_i,
                             const int32_t* site_j, double* out);
/* Lattice of a parameter file: dimension, extents and periodic flags
 * (boundary conditions) of each direction (lib/xml/lattices.xml.in). */
int aed_lattice_geometry(const char* params, int32_t* dim, int32_t* extent, int32_t* periodic);

/* ---- spin-S sectors ----------------------------------------------------- */
/* An Sz sector of the spin model with local spin S = two_s / 2 (1/2 .. 2) on
 * every site: site digits v = m + S in the basis order of basis_states::build
 * (src/alps/model/basisstates.h:175-278, site 0 most significant, Sz
 * ascending per site, lib/xml/models.xml.in:24-36); model->n_up is the
 * digit sum Sz_total + N S (for S = 1/2 the number of up spins).  The
 * Hamiltonian is the spin HAMILTONIAN of models.xml.in:342-373: site terms
 * -h Sz + D Sz^2, bonds Jz Sz Sz + Jxy exchange_xy + K biquadratic (:290-300).
 * FP64; vectors of aed_dimension doubles; aed_solve, aed_eigenvectors and the
 * vector calls take them.  Replaces hamiltonian_matrix::build for local_S > 1/2
 * (hamiltonian_matrix.hpp:402-450); the matrix stays implicit. */
int aed_create_spin(const aed_model_desc* model, int32_t two_s, int device, aed_handle** out);
/* States of rows [offset, offset + count) of a spin-S sector, packed with
 * ceil(log2(2S+1)) bits per site, site 0 most significant. */
int aed_spin_basis(aed_handle* h, uint64_t* states, int64_t offset, int64_t count);

/* ---- momentum sectors --------------------------------------------------- */
/* Translations of a lattice at one momentum k: the identity first. */
typedef struct {
  int32_t n_trans;          /* number of translations (1..62)                          */
  const int32_t* site_map;  /* n_trans x n_sites: translation t moves site i to         *
                             * site_map[t * n_sites + i]                                 */
  const double* phase;      /* n_trans x 2: exp(i k.R_t) as (re, im)                     */
} aed_translations;

/* A momentum sector of the Sz sector of `model`: rows are the representatives
 * of the translation orbits with nonzero weight, vectors are complex, stored
 * as interleaved (re, im) doubles (2 x aed_dimension doubles per vector; the
 * aed_vec_* calls, aed_mult, aed_solve and aed_eigenvectors take them).  FP64.
 * Replaces hamiltonian_matrix::build_basis with TOTAL_MOMENTUM set
 * (src/alps/model/hamiltonian_matrix.hpp:402-417; bloch_basis_states::build,
 * src/alps/model/blochbasisstates.h:92-271) and its matrix elements
 * M(i,j) += val * phase * n_j / n_i (hamiltonian_matrix.hpp:307-345); the
 * matrix stays implicit.  The sector's dimension may be 0. */
int aed_create_momentum(const aed_model_desc* model, const aed_translations* tr, int device, aed_handle** out);
/* Representatives (states as in aed_basis_copy) and normalisations of rows
 * [offset, offset + count) of a momentum sector; either array may be NULL
 * (bloch_basis_states' states and normalization(i)).  A spin-S sector's
 * representatives are 64-bit: states must be NULL (aed_spin_basis lists them). */
int aed_momentum_basis(aed_handle* h, uint32_t* states, double* norms, int64_t offset, int64_t count);
/* A momentum sector of a spin-S Sz sector (local spin S = two_s / 2, the
 * states and Hamiltonian of aed_create_spin): the Bloch basis and matrix
 * elements of aed_create_momentum over the spin-S states (DiagMatrix with
 * TRANSLATION_SYMMETRY for local_S > 1/2).  aed_spin_basis lists its
 * representatives (64-bit packed digits), aed_momentum_basis their
 * normalisations (states NULL); vectors, solves and aed_momentum_expectation
 * as for aed_create_momentum. */
int aed_create_spin_momentum(const aed_model_desc* model, int32_t two_s, const aed_translations* tr, int device,
                             aed_handle** out);
/* Momenta the sparsediag sector loop visits for a parameter file
 * (DiagMatrix::dostep, applications/diag/diag.h:93-114): TOTAL_MOMENTUM when
 * given, else every momentum of lattice.translation_momenta()
 * (src/alps/lattice/hypercubic.h:403-423, the first periodic direction
 * slowest) when TRANSLATION_SYMMETRY (default true), else none.  k: room for
 * `capacity` momenta of n_dirs components, or NULL to query the counts. */
int aed_lattice_momenta(const char* params, int32_t* n_momenta, int32_t* n_dirs, double* k, int32_t capacity);
/* The lattice's translations at momentum k (hypercubic_lattice::translations,
 * hypercubic.h:425-464: the first periodic direction fastest, phase
 * exp(i sum_d shift_d k_d)).  site_map: room for capacity x n_sites entries,
 * phase for capacity x 2; both NULL to query the counts. */
int aed_lattice_translations(const char* params, const double* k, int32_t n_dirs, int32_t* n_trans,
                             int32_t* n_sites, int32_t* site_map, double* phase, int32_t capacity);

/* Replace the couplings of a handle (same N, n_up; any bond list), keeping its
 * basis tables, workspaces and apply tuning: the parameter sweeps sparsediag
 * jobs run (one task per coupling set, applications/diag/diag.h:85-138)
 * without rebuilding the sector.  Rebuilds the coupling tables and the
 * diagonal M(i,i) (hamiltonian_matrix.hpp:422-450). */
int aed_set_couplings(aed_handle* h, const aed_model_desc* model);

/* Sector dimension D (hamiltonian_matrix::dimension). */
int aed_dimension(const aed_handle* h, int64_t* dim);

/* Most recent error message of the calling thread ("" if none). */
const char* aed_last_error(void);

/* Basis states [offset, offset+count) as bit strings (site s <-> bit N-1-s,
 * up = 1), in the reference's order (basisstates.h:175-278).  host_out is host memory. */
int aed_basis_copy(aed_handle* h, uint32_t* host_out, int64_t offset, int64_t count);
/* The state of row idx, widened to 64 bits, for any kind of handle: the bit
 * string of a spin-1/2 Sz sector, the representative of a momentum sector, the
 * packed digits of a spin-S sector (element idx of basis_states, a
 * std::vector of states, src/alps/model/basisstates.h:44-46). */
int aed_basis_state(aed_handle* h, int64_t idx, uint64_t* state);

/* Ranks of `count` host bit strings through the device tables: the row index
 * of each state, or D when the state is outside the sector
 * (basis_states::index, basisstates.h:68-74). */
int aed_index(aed_handle* h, const uint32_t* host_states, int64_t count, int64_t* host_idx);

/* ---- vectors (ietl vectorspace / free functions, src/ietl/vectorspace.h:23-46,
 *      src/ietl/interface/ublas.h:27-55) ------------------------------------ */
int aed_vec_alloc(aed_handle* h, void** dev_vec);          /* zeroed (new_vector)  */
int aed_vec_free(aed_handle* h, void* dev_vec);
int aed_vec_upload(aed_handle* h, void* dev_vec, const double* host);   /* D doubles */
int aed_vec_download(aed_handle* h, const void* dev_vec, double* host); /* D doubles */
int aed_vec_copy(aed_handle* h, const void* x, void* y);               /* ietl::copy  */
int aed_vec_clear(aed_handle* h, void* x);                             /* ietl::clear */
/* ietl::generate with the engine's generator: x[i] = uniform[0,1) from
 * splitmix64(seed, i), bit-identical on host and device. */
int aed_vec_fill_random(aed_handle* h, void* x, uint64_t seed);

/* y = H x (ietl::mult, src/ietl/interface/ublas.h:57-63).  In FP64 every row
 * is summed in ascending column order without FMA contraction, exactly as
 * y = prod(M, x) over the explicit matrix: results are bit-identical to it. */
int aed_mult(aed_handle* h, const void* x, void* y);

int aed_dot(aed_handle* h, const void* x, const void* y, double* out); /* ietl::dot      */
int aed_nrm2(aed_handle* h, const void* x, double* out);               /* ietl::two_norm */
int aed_axpy(aed_handle* h, double a, const void* x, void* y);         /* y += a*x       */
int aed_scal(aed_handle* h, double a, void* x);                        /* x *= a         */
int aed_div(aed_handle* h, double a, void* x);                         /* x /= a         */

/* One fused Lanczos step, lanczos::make_step (src/ietl/lanczos.h:392-406):
 *   w = H v_cur;  alpha = <v_cur, w>;  w -= alpha v_cur;  w -= beta_prev v_prev;
 *   beta = ||w||;  v_next = w / beta.
 * v_prev may be NULL for the first step (lanczos.h:377-390). */
int aed_lanczos_step(aed_handle* h, const void* v_prev, const void* v_cur, void* v_next,
                     double beta_prev, double* alpha, double* beta);

/* ---- whole solves ----------------------------------------------------------- */
typedef struct {
  int32_t nev;          /* NUMBER_EIGENVALUES (>= 1)                                  */
  int32_t max_iter;     /* MAX_ITERATIONS, 0 = min(10 D, 1000)                         */
  double rtol, atol;    /* lanczos_iteration_nlowest tolerances, 0 = 100 eps (iteration.h:110-113) */
  uint64_t seed;        /* start-vector seed                                           */
  const double* start;  /* optional HOST start vector (D doubles), else seeded          */
  int32_t refine;       /* AED_FP32 handles: 0 = mixed: FP32 Lanczos, then FP64
                           Rayleigh-Ritz over its Ritz vectors, FP64 Lanczos from them
                           when the Rayleigh-Ritz error bound is not met (default);
                           1 = mixed with the FP64 Lanczos refinement only;
                           -1 = plain FP64 Lanczos on the same handle                  */
  int32_t profile;      /* 1: time every apply with CUDA events (res->apply_ms)         */
  int32_t resume;       /* 1: continue the handle's live FP64 recurrence (the last solve's
                           or one aed_lanczos_load restored) until the stop rule holds
                           for nev values: ietl's more_eigenvalues (lanczos.h:77-78);
                           start / seed / refine are then ignored                      */
  int32_t reorth;       /* 1: full reorthogonalisation of the mixed path's FP32 Lanczos
                           vectors against the stored basis (classical Gram-Schmidt,
                           twice, FP64 sums) each step; AED_FP32 handles, refine 0 or 1.
                           An engine option: ietl's lanczos has no reorthogonalisation */
} aed_solve_opts;

#define AED_MAX_NEV 16
typedef struct {
  int32_t n_evals;              /* min(nev, #distinct non-ghost values) (sparsediag.h:115-118) */
  int32_t iterations;           /* T-matrix size at convergence (FP64 phase for FP32 handles;
                                   the number of FP64 applies when refined_by is
                                   AED_REFINE_RAYLEIGH_RITZ)                                     */
  int32_t iterations_low;       /* FP32 phase iterations (0 for FP64 handles)                    */
  int32_t converged;            /* 1 when all nev errors met the tolerance                       */
  double evals[AED_MAX_NEV];    /* lowest distinct eigenvalues, ascending                        */
  double errors[AED_MAX_NEV];   /* |beta_m z_{m,i}| error estimates (tmatrix.h:159-183); for
                                   AED_REFINE_RAYLEIGH_RITZ the bound on lambda_i's error     */
  double evals_low[AED_MAX_NEV];/* FP32-phase eigenvalues before refinement (FP32 handles)       */
  double seconds;               /* wall time of the solve                                        */
  double apply_ms;              /* mean device time of one H*x inside the solve                  */
  int32_t refined_by;           /* FP32 handles: how the FP32 values were refined (AED_REFINE_*) */
} aed_solve_result;

#define AED_REFINE_NONE 0           /* an FP64 solve                                         */
#define AED_REFINE_RAYLEIGH_RITZ 1  /* FP64 Rayleigh-Ritz over the FP32 Ritz vectors          */
#define AED_REFINE_LANCZOS 2        /* FP64 Lanczos from the FP32 Ritz vectors                */

/* Lanczos eigenvalues: SparseDiagMatrix::do_subspace's Lanczos part
 * (applications/diag/sparsediag/sparsediag.h:104-118) with ietl::lanczos
 * (src/ietl/lanczos.h:341-406), lanczos_iteration_nlowest (src/ietl/iteration.h:106-130)
 * and Tmatrix::compute's distinct/ghost rules (src/ietl/tmatrix.h:121-228). */
int aed_solve(aed_handle* h, const aed_solve_opts* opts, aed_solve_result* res);

/* Ritz vectors (lanczos::eigenvectors, src/ietl/lanczos.h:134-336) of the k
 * lowest distinct eigenvalues of the last aed_solve (or resumed solve): its
 * FP64 recurrence is run again from the same start -- `opts` must give the
 * solve's seed or start vector; a mixed solve's FP64 phase restarts from the
 * vector the handle kept -- and psi_i = sum_j z_i[j] v_j accumulates in FP64.
 * The replayed alpha/beta must equal the solve's bit for bit
 * (lanczos.h:248-250,266-268; AED_ERR_MISMATCH otherwise).  vecs[i]: device
 * vectors of the handle (FP32 handles receive psi rounded to FP32); evals[i]
 * and residuals[i] = |H psi_i - lambda_i psi_i| (lanczos.h:284-295), both
 * optional.  The FP64 apply is used for AED_FP32 handles as well. */
int aed_eigenvectors(aed_handle* h, const aed_solve_opts* opts, int32_t k, void* const* vecs, double* evals,
                     double* residuals);

/* Checkpoint of the live FP64 Lanczos recurrence: Tmatrix::save and
 * lanczos::save (src/ietl/tmatrix.h:66-77, src/ietl/lanczos.h:86-98) -- alpha,
 * beta, v_{m-1}, v_m and the step count -- into a host buffer of
 * aed_lanczos_state_bytes bytes (0 when no recurrence is live).  A load
 * checks that the state belongs to the same Hamiltonian (sector and
 * couplings); an aed_solve with opts.resume = 1 then continues it. */
int aed_lanczos_state_bytes(aed_handle* h, int64_t* bytes);
int aed_lanczos_save(aed_handle* h, void* buf, int64_t bytes);
int aed_lanczos_load(aed_handle* h, const void* buf, int64_t bytes);

/* Copy the alpha/beta recurrence of the last aed_solve (FP64 phase; a mixed
 * solve refined by Rayleigh-Ritz has none and gives its FP32 phase) to host;
 * *n receives its length (at most cap entries are written). */
int aed_last_tmatrix(aed_handle* h, double* alpha, double* beta, int32_t cap, int32_t* n);
/* The same for the FP32 phase of the last mixed solve of an AED_FP32 handle.
 * Engine addition, no reference counterpart. */
int aed_last_tmatrix_fp32(aed_handle* h, double* alpha, double* beta, int32_t cap, int32_t* n);

/* Tmatrix::compute(true) on a host recurrence (src/ietl/tmatrix.h:121-228):
 * distinct non-ghost eigenvalues of T (alpha[0..n), beta[0..n-1) off-diagonal,
 * beta[n-1] = beta_{m+1}), their error estimates |beta_{m+1} z_{m,i}| and
 * multiplicities; at most cap written, *count = how many.  Host-only. */
int aed_tmatrix(int32_t n, const double* alpha, const double* beta, int32_t cap, double* evals, double* errors,
                int32_t* mults, int32_t* count);

/* Time `reps` back-to-back applies y = H x on the handle's stream with CUDA
 * events; *ms = mean milliseconds per apply. */
int aed_time_mult(aed_handle* h, const void* x, void* y, int32_t reps, double* ms);

/* As aed_time_mult, for apply variant `variant` (-1: the handle's tuned one),
 * with the per-tile <x, y> partials of the fused Lanczos step when
 * with_alpha != 0.  *variant_used receives the variant timed. */
int aed_time_apply(aed_handle* h, const void* x, void* y, int32_t reps, int32_t variant, int32_t with_alpha,
                   double* ms, int32_t* variant_used);

/* Apply variants (the kernel shapes that the autotuner times on a handle's
 * first apply): their number, and the name of variant `variant` (NULL when out
 * of range).  Engine addition, no reference counterpart. */
int32_t aed_apply_variant_count(void);
const char* aed_apply_variant_name(int32_t variant);

/* ---- batched / served solves ------------------------------------------------
 * Many independent requests (a model and solve options each) advance together
 * on one GPU: every engine step runs one Lanczos step of every resident
 * request over work queues of (request, tile) and (request, chunk) items, and
 * a CUDA graph holds S steps plus the convergence check.  Requests are
 * admitted in arrival order while their HBM footprint fits the server's
 * budget, and join the running batch at the next step (continuous batching).
 * The analogue of the reference's task farm over independent parameter sets
 * (src/alps/scheduler/mpp_scheduler.C:50) on one GPU.  AED_FP32 servers run
 * the mixed path (FP32 Lanczos basis, FP64 refinement to r^2/gap <= 1e-11
 * |lambda|); AED_FP64 servers the plain FP64 recurrence with the ietl rule,
 * checked every S steps (results come from T at the first check after
 * convergence).  A request's result does not depend on the other requests in
 * the batch. */
typedef struct aed_server aed_server;

typedef struct {
  int32_t device;
  int32_t max_slots;         /* resident requests at most (default 512)                */
  int32_t steps_per_launch;  /* S, Lanczos steps per graph launch (default 8)          */
  int32_t precision;         /* AED_FP32 (mixed) or AED_FP64                           */
  double hbm_fraction;       /* budget as a fraction of free memory (default 0.8)      */
  int64_t hbm_budget_bytes;  /* explicit budget in bytes (overrides hbm_fraction)      */
  int64_t reserve_bytes;     /* device memory mapped into the server's pool at creation
                                (-1: the whole budget; 0: none), so that requests do not
                                pay for mapping fresh memory on first use               */
  int32_t max_lanes;         /* requests of dimension >= lane_min_dim run as single-instance
                                solves (their own handle, stream and host thread, the
                                fastest apply variants) beside the batch, at most this
                                many at once (default 2)                                  */
  int64_t lane_min_dim;      /* 0: default 2^21; -1: no lanes (every request batched)    */
} aed_server_opts;

typedef struct {
  int32_t resident, queued;
  int64_t bytes_used, bytes_budget;
  int64_t graph_launches;
  int32_t lanes;             /* single-instance solves running                           */
} aed_server_stats;

int aed_server_create(const aed_server_opts* opts, aed_server** out);
int aed_server_destroy(aed_server* s);
/* Queue a request.  AED_ERR_ADMISSION if its footprint alone exceeds the budget.
 * opts->start and opts->resume are ignored (start vectors are drawn from
 * opts->seed). */
int aed_server_submit(aed_server* s, const aed_model_desc* model, const aed_solve_opts* opts, int64_t* ticket);
/* Admit what fits, run one graph launch (S engine steps + check), harvest
 * finished requests.  *n_pending = resident + queued requests afterwards. */
int aed_server_step(aed_server* s, int32_t* n_pending);
/* AED_PENDING while running; AED_OK with *out filled (out->seconds = latency
 * from submission to completion) once, after which the ticket is forgotten. */
int aed_server_poll(aed_server* s, int64_t ticket, aed_solve_result* out);
int aed_server_cancel(aed_server* s, int64_t ticket);
int aed_server_get_stats(aed_server* s, aed_server_stats* out);

/* Copy v_j (D floats, device memory) of the FP32 Lanczos basis that the last
 * mixed solve of an AED_FP32 handle stored, j < iterations_low + 1: for
 * checking the basis (orthogonality, with and without opts.reorth).  Engine
 * addition, no reference counterpart (ietl keeps no basis). */
int aed_lanczos_vector(aed_handle* h, int32_t j, void* out);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own
 * work or record timing events on it.  Engine addition, no reference counterpart. */
int aed_get_stream(aed_handle* h, void** stream);

/* Number of engine kernel launches made by this process so far. */
int aed_launch_count(int64_t* count);

/* Dot product that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory: applications
 * whose device memory belongs to another allocator (a framework's caching
 * allocator, a fixed arena given to a simulation code at start-up), and
 * latency-critical loops that cannot pay for cudaMalloc/cudaFree (cudaFree
 * synchronises the whole device).
 *
 * *out (a device double) = sum_i x[i] * y[i] over n device elements (double for
 * AED_FP64, float for AED_FP32, accumulated in double), with the same chunking
 * and summation order as aed_dot, so both return the same bits.  Work is
 * queued on `stream` (a cudaStream_t; NULL = the legacy default stream) and the
 * call returns without waiting.  The caller passes the inputs and the output;
 * the scratch (the per-chunk partial sums) is a fixed 512 KiB device array
 * inside libaed.so that every GPU loading the library keeps until the process
 * exits, so n is limited to 268,435,456 elements (larger n: AED_ERR_INVALID,
 * nothing launched).  The first call on a device looks up that array's device
 * address; make that first call before any stream capture.  That address is
 * kept for the life of the process: after a cudaDeviceReset of that device
 * (which unloads the library's module there) it is stale, so do not call
 * aed_dot_noalloc on a device that was reset.  Every call
 * overwrites the partials it then reads, so nothing needs clearing, but all
 * calls share the one array: calls that overlap on the GPU (different
 * streams, different host threads) race and can return wrong sums; order
 * them on one stream. */
int aed_dot_noalloc(const void* x, const void* y, int64_t n, int precision, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AED_H */
