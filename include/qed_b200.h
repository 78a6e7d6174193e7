/*
 * qed_b200.h -- C ABI of the B200 exact-diagonalization (ED) impurity solver.
 *
 * This is the drop-in boundary for pyqcm's cluster ground-state and cluster
 * Green-function path. Each entry point below names the reference interface
 * it replaces (paths relative to the pyqcm source tree). The reference's ED
 * layer is the C++ namespace ED (src_ed/qcm_ED.hpp:23-340); its inner plugin
 * point is the Hamiltonian<HilbertField> interface
 * (src_ed/Hamiltonian/Hamiltonian_base.hpp:43-82), chosen per sector by
 * model_instance::create_hamiltonian (src_ed/model_instance.hpp:193-238).
 *
 * Conventions
 *  - Every function returns a status code (QED_OK == 0). On failure the
 *    message is available from qed_last_error() (per thread). The C++ adapter
 *    rethrows a non-zero status as qcm_error, matching qcm_ED_throw
 *    (src_util/parser.cpp:323-328).
 *  - Orbital indices are 0-based: orbital i < n_orb is spin up, i + n_orb is
 *    spin down (n_orb = n_sites + n_bath), as in the reference's operators
 *    after its Python binding subtracts 1 (src_python/qcm_ED_wrap.hpp:199-200).
 *  - Complex numbers are interleaved (re, im) doubles. Matrices are
 *    column-major, like the reference's matrix<T> (src_util/matrix.cpp:11-16).
 *  - All array arguments are host memory owned by the caller, except where a
 *    function name ends in _device (device pointers on the current device).
 *  - Device memory is owned by the instance / Hamiltonian handles and freed by
 *    qed_erase_model_instance / qed_hamiltonian_destroy. No device pointer
 *    owned by the library escapes it.
 *  - Thread safety: calls on different instance labels may run concurrently;
 *    calls on one label are serialised internally.
 */
#ifndef QED_B200_H
#define QED_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QED_OK 0
#define QED_ERR_ARGUMENT 1      /* bad argument, unknown name/label, invalid sector       */
#define QED_ERR_LANCZOS 2       /* Lanczos iteration cap (src_ed/Hamiltonian/Lanczos.hpp:92) */
#define QED_ERR_QMATRIX 3       /* Q-matrix norm check (src_ed/Q_matrix.hpp:255-259)         */
#define QED_ERR_CUDA 4          /* CUDA runtime error                                       */
#define QED_ERR_MEMORY 5        /* device memory budget exceeded                            */
#define QED_ERR_UNSUPPORTED 6   /* model outside this solver's scope (e.g. anomalous, complex) */
#define QED_ERR_NO_DEVICE 7     /* no CUDA device / extension not usable                    */
#define QED_ERR_INTERNAL 8

/* Copies the last error message of the calling thread; returns its length. */
int qed_last_error(char *buf, int len);
/* No counterpart in the reference: the launch shapes the H.v autotuner picked so
 * far, one JSON object per sector shape (dim_up, dim_dn) with the shape chosen,
 * whether every candidate wrote the same bits of H x (bit_identical) and the time
 * of every candidate (ms per H.v). Writes at most len - 1 bytes
 * and a terminating 0; returns the full length. */
int qed_hv_tuning_report(char *buf, int len);
/* No counterpart in the reference: diagnostics of the window H.v kernels of
 * large sectors (host only, no device needed). qed_window_plan plans the windows
 * of one spin (L sites, N particles, npairs directed hopping pairs pd[q] <- ps[q]
 * of amplitude amp[q]) and, when they fit, applies the window form of that
 * spin's hop operator to x (C(L, N) doubles in basis order) on the host into y;
 * *nwindows = 0 when the pairs do not fit windows. qed_window_compile compiles
 * the window kernels of a sector whose two spins have those pairs (N_up, N_dn
 * particles) with NVRTC and writes its log (ptxas registers and spills) to buf;
 * *ok = 1 on success. */
int qed_window_plan(int L, int N, int npairs, const int *pd, const int *ps, const double *amp, const double *x,
                    double *y, int *nwindows);
int qed_window_compile(int L, int n_up, int n_dn, int npairs, const int *pd, const int *ps, char *buf, int len,
                       int *ok);
/* Number of H.v calls that ran the window kernels so far in this process. */
int qed_window_launches(long long *n);
/* No counterpart in the reference: one spin's tables as this solver builds them
 * (host computation, no device needed), for checks of the hop rule of
 * HS_half_operator (src_ed/Operators/HS_half_operator.hpp:17-45). t and vsame:
 * L x L row-major one-body matrix and same-spin density-density terms. Writes
 * dim = C(L, N) strings (increasing), cnt and diag, *width entries per string
 * of the ELL table into ell (entry k of string i at ell[k * dim + i] = rank << 8
 * | value slot; at most ell_capacity entries) and *nvals value slots into vals
 * (at most 258). bank_order != 0 returns the bank-ordered table. */
int qed_spin_table_host(int L, int N, const double *t, const double *vsame, int bank_order, unsigned *bits,
                        unsigned char *cnt, double *diag, unsigned *ell, long ell_capacity, int *width,
                        double *vals, int *nvals);

/* Selects the CUDA device used by this process (default 0). */
int qed_init(int device);

/* Global options, same names and defaults as the reference's QCM initialisation
 * (src_util/global_parameter.cpp:10-92; setters src_util/global_parameter.hpp:74-77).
 * The get variants return QED_ERR_ARGUMENT for an unknown name. */
int qed_set_global_int(const char *name, long value);
int qed_set_global_double(const char *name, double value);
int qed_set_global_char(const char *name, char value);
int qed_set_global_bool(const char *name, int value);
int qed_get_global_double(const char *name, double *value);

/* ED::new_model (src_ed/qcm_ED.hpp:33) without generators (trivial point group,
 * the spin-factorized basis; models with generators: qed_new_model_generators). */
int qed_new_model(const char *name, int n_sites, int n_bath);

/* ED::new_operator (src_ed/qcm_ED.hpp:56), real elements. type is "one-body"
 * or "interaction". Elements (r[k], c[k], v[k]) follow the reference: one-body
 * elements with r > c are ignored and r < c ones get their Hermitian partner
 * (src_ed/Operators/one_body_operator.hpp:63-71); interaction elements are
 * ordered r <= c (src_ed/Operators/interaction_operator.hpp:45-50). */
int qed_new_operator(const char *model, const char *name, const char *type, int n, const int *r,
                     const int *c, const double *v);

/* ED::new_model_instance (src_ed/qcm_ED.hpp:80). sectors: "R0:N8:S0[/...]". */
int qed_new_model_instance(const char *model, int n, const char **names, const double *values,
                           const char *sectors, int label);

/* ED::erase_model_instance (src_ed/qcm_ED.cpp:65-68). Frees device memory. */
int qed_erase_model_instance(int label);

/* ED::mixing (src_ed/qcm_ED.hpp:92): 0 normal, 4 up-down. */
int qed_mixing(int label, int *mixing);

/* ED::ground_state_solve (src_ed/qcm_ED.hpp:104 -> model_instance::low_energy_states,
 * src_ed/model_instance.hpp:245-347). Returns the GS energy and the sector
 * string of the kept states ("R0:N8:S0:1" style, as GS_string()). */
int qed_ground_state_solve(int label, double *energy, char *sectors, int len);

/* Batched ground states (the per-instance loop of the lattice layer,
 * src_qcm/lattice_model_instance.cpp:107-113, run by OpenMP threads there):
 * solves the instances labels[0..n) concurrently on `threads` host threads
 * (0 = hardware concurrency, capped at 64), each driving its own CUDA stream.
 * energies[i] receives the ground-state energy of labels[i]. Every instance is
 * attempted; the status of the first failure is returned (message via
 * qed_last_error). */
int qed_ground_state_solve_batch(const int *labels, int n, int threads, double *energies);

/* Batched Green_function_solve over labels[0..n), same threading rules. */
int qed_Green_function_solve_batch(const int *labels, int n, int threads);

/* No counterpart in the reference (its batching is the OpenMP loop of the
 * lattice layer): the batched solves as an asynchronous work queue. A batch of
 * instances is handed to a background host thread, which runs
 * qed_ground_state_solve_batch (what = QED_BATCH_GROUND_STATE) or
 * qed_Green_function_solve_batch (QED_BATCH_GREEN_FUNCTION: ground states
 * first where needed) on `threads` threads; the call returns at once with a
 * ticket (> 0). While the batch runs, other calls on its instances wait for
 * it (each instance is locked for the batch); results are then read through
 * the per-instance entries (qed_ground_state_solve returns the solved state).
 * Batches run concurrently with one another, each on its own streams. */
#define QED_BATCH_GROUND_STATE 1
#define QED_BATCH_GREEN_FUNCTION 2
int qed_batch_submit(const int *labels, int n, int what, int threads, long long *ticket);
/* *done = 0 while the batch runs (returns QED_OK); once it has finished,
 * *done = 1, the ticket is released and the batch's status is returned (its
 * first failure's message via qed_last_error). Unknown ticket: QED_ERR_ARGUMENT. */
int qed_batch_poll(long long ticket, int *done);
/* As qed_batch_poll, after waiting up to timeout_ms milliseconds for the
 * batch to finish (timeout_ms < 0: without limit). */
int qed_batch_wait(long long ticket, int timeout_ms, int *done);

/* ED::Green_function_solve (src_ed/qcm_ED.hpp:122 -> src_ed/model_instance.hpp:517-555):
 * band-Lanczos Q-matrix (GF_method 'L') or continued fractions ('F'). */
int qed_Green_function_solve(int label);

/* ED::Green_function_dimension (src_ed/qcm_ED.hpp:241). */
int qed_Green_function_dimension(int label, int *dim);

/* ED::Green_function (src_ed/qcm_ED.hpp:134 -> src_ed/model_instance.hpp:566-635),
 * batched over nz frequencies z (interleaved complex). G receives nz blocks of
 * dim x dim complex, column-major, evaluated on the GPU. */
int qed_Green_function(int label, int spin_down, int nz, const double *z, double *G);

/* The wavevector sum of the self-energy-functional integrand on a fixed grid, per
 * frequency: lattice_model_instance::SEF_integrand_k (src_qcm/lattice_model_instance.cpp:618-640)
 * under QCM::k_integral_grid (src_util/integrate.cpp:177-240), as Potthoff_functional's
 * discrete-grid path uses them (src_qcm/lattice_model_instance.cpp:520-545).
 * For each of the nw frequencies w[i] (the point i*w[i] on the imaginary axis):
 *   I_w[i] = 1/Nk sum_k log |det(V(k) G(i w[i]) - 1)|,  k = (a/nkx, b/nky, c/nkz),
 *   V(k) = V0 + sum_e v[e] exp(2 pi i k.R[e]) at row r[e], column c[e]   (set_V, src_qcm/CPT.cpp:22-64),
 * with G the cluster Green function of ED instance `label` (spin_down selects the
 * down block under up_down mixing), V0 dim x dim complex column-major (the
 * k-independent part of V), R[3 e..3 e + 2] integer superlattice coordinates and
 * v[e] complex (interleaved). G and the nw x Nk determinants are computed on the GPU;
 * dim (at most 16) must be the cluster's Green-function dimension. */
int qed_sef_integrand_grid(int label, int spin_down, int dim, const double *V0, int nel, const int *r, const int *c,
                           const int *R, const double *v, int nw, const double *w, int nkx, int nky, int nkz,
                           double *I_w);

/* The projected CPT Green function of the CDMFT host, per frequency:
 * lattice_model_instance::projected_Green_function (src_qcm/CPT.cpp:283-346) with
 * set_Gcpt (:76-86) and set_V (:22-64): Gproj(i w[i]) = average over the grid
 * k = ((a + offset)/nkx, (b + offset)/nky, (c + offset)/nkz) of G (1 - V(k) G)^{-1},
 * V(k) = V0_i + sum_e v[e] exp(2 pi i k.R[e]). V0: nw k-independent parts (dim x dim
 * complex column-major each; with bath orbitals they hold -Gamma(i w[i])), elements as
 * in qed_sef_integrand_grid; Gproj: nw dim x dim complex, column-major. The reference's
 * grid is kgrid_side points per direction with offset 0.5. On the GPU; dim <= 16. */
int qed_cpt_projected_green_function(int label, int spin_down, int dim, const double *V0, int nel, const int *r,
                                     const int *c, const int *R, const double *v, int nw, const double *w,
                                     int nkx, int nky, int nkz, double offset, double *Gproj);

/* ED::self_energy (src_ed/qcm_ED.hpp:180 -> src_ed/model_instance.hpp:683-700), batched. */
int qed_self_energy(int label, int spin_down, int nz, const double *z, double *S);

/* ED::hybridization_function (src_ed/qcm_ED.hpp:210 -> src_ed/model_instance.hpp:1004-1018), batched. */
int qed_hybridization_function(int label, int spin_down, int nz, const double *z, double *H);

/* ED::Green_function_average (src_ed/qcm_ED.hpp:146): <c^+_b c_a>, d x d complex,
 * d from qed_Green_function_average_dimension: the number of cluster sites, or
 * cluster + bath orbitals for an uncorrelated instance (as the reference returns). */
int qed_Green_function_average(int label, int spin_down, double *M);
int qed_Green_function_average_dimension(int label, int *d);

/* ED::cluster_averages (src_ed/qcm_ED.hpp:113 -> src_ed/model_instance.hpp:149-173,
 * 340-345): for each operator of the instance, in name order, its ground-state
 * average and variance (divided by the number of sites for cluster operators).
 * cap is the capacity of ave and var; *n receives the number of operators;
 * names receives the operator names, each followed by '\n', in a buffer of
 * names_size bytes. Solves the ground state first if needed. */
int qed_cluster_averages(int label, int cap, int *n, double *ave, double *var, char *names, int names_size);

/* ED::model_size (src_ed/qcm_ED.hpp:42): sites, bath orbitals, group elements (1). */
int qed_model_size(const char *model, int *n_sites, int *n_bath, int *n_elements);

/* ED::exists (src_ed/qcm_ED.hpp:66): *found = 1 if the model has the operator. */
int qed_operator_exists(const char *model, const char *op, int *found);

/* ED::matrix_elements (src_ed/qcm_ED.hpp:308): the operator's type ("one_body" or
 * "interaction", into a buffer of type_size bytes) and its stored elements
 * (r, c, v) after the reference's normalisation; cap is the capacity of r, c, v. */
int qed_matrix_elements(const char *model, const char *op, char *type, int type_size, int cap, int *n, int *r,
                        int *c, double *v);

/* ED::complex_HS (src_ed/qcm_ED.hpp:94): always 0 (real Hilbert space). */
int qed_complex_HS(int label, int *flag);

/* ED::Green_function_density (src_ed/qcm_ED.hpp:152): the density from the
 * solved Green function (0 before Green_function_solve). */
int qed_Green_function_density(int label, double *density);

/* ED::hopping_matrix (src_ed/qcm_ED.hpp:174): the cluster one-body matrix,
 * n_sites x n_sites complex, column-major (spin down only differs for up_down mixing). */
int qed_hopping_matrix(int label, int spin_down, double *H);

/* ED::hopping_matrix_full (src_ed/qcm_ED.hpp:175): cluster + bath one-body matrix,
 * d x d complex with d = n_sites + n_bath (written to *d), column-major; diag
 * selects the diagonalised bath. H may be NULL to query d. */
int qed_hopping_matrix_full(int label, int spin_down, int diag, int *d, double *H);

/* ED::interactions (src_ed/qcm_ED.hpp:180): (r, c, v * value) for every element of
 * the instance's interaction operators; cap is the capacity of r, c, v. */
int qed_interactions(int label, int cap, int *n, int *r, int *c, double *v);

/* ED::tr_sigma_inf (src_ed/qcm_ED.hpp:252): trace of the self-energy at infinite
 * frequency, extrapolated from three large imaginary frequencies. */
int qed_tr_sigma_inf(int label, double *value);

/* ED::susceptibility (src_ed/qcm_ED.hpp:202 -> src_ed/model_instance.hpp:1027-1061):
 * the dynamical susceptibility of operator op at nw complex frequencies w
 * (re, im pairs) into chi (re, im pairs). */
int qed_susceptibility(int label, const char *op, int nw, const double *w, double *chi);

/* ED::susceptibility_poles (src_ed/qcm_ED.hpp:213 -> src_ed/model_instance.hpp:1070-1115):
 * poles (e > 1e-8) and residues (> 1e-6) of the susceptibility, poles closer
 * than 1e-4 merged; cap is the capacity of e and r. */
int qed_susceptibility_poles(int label, const char *op, int cap, int *n, double *e, double *r);

/* ED::fidelity (src_ed/qcm_ED.hpp:244 -> src_ed/model_instance.hpp:1258-1271): the sum
 * over state pairs of the two instances in the same sector of w1 w2 |<psi1|psi2>|^2. */
int qed_fidelity(int label1, int label2, double *fidelity);

/* ED::Potthoff_functional (src_ed/qcm_ED.hpp:222; SEF_bath + E0, src_ed/qcm_ED.cpp:330-334). */
int qed_Potthoff_functional(int label, double *omega);

/* ED::qmatrix (src_ed/qcm_ED.hpp:286 -> src_ed/model_instance.hpp:1425-1451).
 * On entry *M is the capacity of e (and of v, in columns); on exit the number
 * of poles. v is L x M complex, column-major. */
int qed_qmatrix(int label, int spin_down, int *M, int *L, double *e, double *v);

/* Continued-fraction coefficients (GF_method 'F') of the first state for the
 * pair (o1, o2), o2 <= o1, electron (pm = +1) or hole (pm = -1); the
 * continued_fraction a/b arrays of src_ed/continued_fraction.cpp:33-39.
 * On entry *n is the capacity; on exit the number of levels. */
int qed_cf_coefficients(int label, int spin_down, int o1, int o2, int pm, int *n, double *a,
                        double *b);

/* ---- instance checkpoints ----------------------------------------------------
 * The data of model_instance::write_hdf5 / read_hdf5 (src_ed/model_instance.hpp:1339-1421,
 * state.hpp:52-115, Q_matrix.hpp:321-345, continued_fraction_set.cpp:136-176),
 * behind ED::write_instance_hdf5 / ED::read_instance_hdf5 (src_ed/qcm_ED.cpp:373-403).
 * The HDF5 file itself is written and read by the caller (pyqcm_b200/hdf5.py).
 * gf_format: 0 Q-matrices ("bl"), 1 continued fractions ("cf"), 2 matrix
 * continued fractions ("mcf", not supported here). Trivial point group only. */
/* Solves the Green function if needed (as write_hdf5 does), then: state count,
 * GS energy, GS sector string, GF format and mixing. */
int qed_instance_states(int label, int *n_states, double *gs_energy, char *gs_sectors, int len, int *gf_format,
                        int *mixing);
/* Parameter values of the instance: names separated by '\n' in names (capacity
 * names_size), values[cap]; *n the count. */
int qed_instance_parameters(int label, int cap, int *n, char *names, int names_size, double *values);
/* State i: sector string, energy, weight. */
int qed_instance_state(int label, int i, char *sector, int len, double *energy, double *weight);
/* Q-matrix of state i: L x M residues v (column-major, sqrt(weight) included) and
 * poles e; with e == NULL only L and M. */
int qed_instance_state_qmatrix(int label, int i, int spin_down, int cap, int *L, int *M, double *e, double *v);
/* Continued fraction (o1, o2), o2 <= o1, electron (pm = +1) or hole (pm = -1) of
 * state i: levels a[n], b[n]; with a == NULL only n. */
int qed_instance_state_cf(int label, int i, int spin_down, int o1, int o2, int pm, int cap, int *n, double *a,
                          double *b);
/* Loading (read_hdf5): begin (drops the instance's states), one load_state per
 * state (its index returned), its Q-matrices or continued fractions, then end:
 * the instance is then solved, with Green_function_average and the density
 * computed from the loaded data as the reference does after reading. */
int qed_instance_load_begin(int label, double gs_energy, int gf_format, int mixing);
int qed_instance_load_state(int label, const char *sector, double energy, double weight, int *index);
int qed_instance_load_qmatrix(int label, int i, int spin_down, int L, int M, const double *e, const double *v);
int qed_instance_load_cf(int label, int i, int spin_down, int o1, int o2, int pm, int n, const double *a,
                         const double *b);
int qed_instance_load_end(int label);

/* Ground-state vector of the first kept state (factorized layout
 * psi[up_rank + dim_up * dn_rank], src_ed/ED_basis.cpp:142-165).
 * *dim receives the dimension; psi may be NULL to query it. */
int qed_ground_state_vector(int label, long *dim, double *psi);

/* ---- plugin point: the Hamiltonian of one sector --------------------------
 * Hamiltonian<double> (src_ed/Hamiltonian/Hamiltonian_base.hpp:43-82) realised
 * on the device in spin-factorized form (replaces Hamiltonian_Factorized,
 * src_ed/Hamiltonian/Hamiltonian_Factorized.hpp:32-87). */
typedef struct qed_hamiltonian qed_hamiltonian;

int qed_hamiltonian_create(int label, const char *sector, qed_hamiltonian **h, long *dim);
/* y += H x with host vectors (Hamiltonian::mult_add). */
int qed_hamiltonian_mult_add(qed_hamiltonian *h, const double *x, double *y);
/* y = H x with device vectors on the current device, enqueued on `stream`
 * (a cudaStream_t; NULL is the legacy default stream, as in the CUDA runtime).
 * Asynchronous: returns after the launches are enqueued. */
int qed_hamiltonian_apply_device(qed_hamiltonian *h, const double *x, double *y, void *stream);
/* y = H x fused with the reductions a Lanczos step needs (LanczosEigenvalue,
 * src_ed/Hamiltonian/Lanczos.hpp:68-77, takes <v, Hv> and norms right after
 * mult_add): dots[0] = <x, y>, dots[1] = <y, y>, dots[2] = <x, x>, written to
 * the device array `dots` (3 doubles). Enqueued on `stream` (NULL = legacy
 * default stream); the per-block partial sums live in a buffer the handle
 * allocates with cudaMalloc on its first call. */
int qed_hamiltonian_apply_dots_device(qed_hamiltonian *h, const double *x, double *y, double *dots,
                                      void *stream);
/* Same result as qed_hamiltonian_apply_dots_device, but the call allocates no
 * memory at all: no cudaMalloc, cudaFree or allocating library routine. It has
 * no counterpart in the reference; it exists for callers that cannot allocate
 * device memory when they call in, e.g. a process whose device memory belongs
 * to another runtime's pool, or a loop that cannot afford cudaMalloc's implicit
 * device synchronisation. The caller passes x, y and dots (3 doubles) in device
 * memory; the per-block partial sums live in a fixed 682 KB array compiled into
 * the library (1184 rows), which every GPU that loads the library holds until
 * the process exits. A Hamiltonian whose column pass would need more rows than
 * that is rejected with QED_ERR_MEMORY (never on a 148-SM B200). The first call
 * on a device looks up the array's device address; make that first call before
 * any stream capture. All calls share the array: calls that overlap on the GPU
 * (different streams, no ordering between them) race and give wrong sums; a
 * call leaves nothing that a later call depends on. */
int qed_hamiltonian_apply_dots_device_noalloc(qed_hamiltonian *h, const double *x, double *y,
                                              double *dots, void *stream);
/* Hamiltonian::diag (src_ed/Hamiltonian/Hamiltonian_base.hpp:57). */
int qed_hamiltonian_diag(qed_hamiltonian *h, double *d);
int qed_hamiltonian_destroy(qed_hamiltonian *h);

/* ---- basis (ED_halfbasis, src_ed/ED_basis.cpp:115-135) ---------------------
 * All L-bit strings with N set bits in ascending order, generated on the GPU by
 * unranking in the combinatorial number system (bit-exact with the sorted list). */
int qed_halfbasis(int L, int N, unsigned *strings, long *dim);
/* Rank of each string (ED_halfbasis::index; returns dim for a string not in the
 * basis), computed on the GPU. */
int qed_halfbasis_rank(int L, int N, long n, const unsigned *strings, unsigned *ranks);

/* c_a applied to every basis state of sector (N_up, N_dn) (Destroy,
 * src_ed/ED_basis.cpp:79-110), computed on the GPU: target index (or -1) and
 * fermion phase bit per source state. */
int qed_destroy_table(int L, int n_up, int n_dn, int a, long *target, int *phase);

/* ---- Cluster point group -----------------------------------------------------
 * The Abelian point group of a cluster model (symmetry_group,
 * src_ed/symmetry_group.hpp:38-92), built from generators given as
 * ED::new_model (src_ed/qcm_ED.hpp:34) takes them: n_gen rows of n_sites + n_bath
 * 0-based entries, site entries a permutation, bath entries orbital labels or,
 * with bath_irrep, phases in units of 2 pi / g. Host logic (no device work);
 * the kernels evaluate the same per-state maps. Errors carry the reference's
 * messages (invalid or non-commuting generators). */

/* ED::new_model with symmetry generators (src_ed/qcm_ED.hpp:34; the reference's
 * Python binding converts pyqcm's 1-based generators to this 0-based form,
 * src_python/qcm_ED_wrap.hpp:145-163). The group is checked and kept with the
 * model; sector strings of its instances may name irreps R0..R(g-1). Their
 * ground states and Green functions are solved in the symmetry-adapted basis:
 * per-irrep sector solves, per-irrep band-Lanczos Q-matrices of the symmetric
 * orbitals, consolidated in the site basis as Q_matrix_set::consolidated_qmatrix
 * (src_ed/Q_matrix_set.hpp:144-163) does. QED_ERR_UNSUPPORTED for groups with
 * complex characters (a generator of order above 2) and for continued-fraction
 * Green functions (GF_method 'F') of such models. The sectors' Hamiltonians are
 * also available through qed_mixed_hamiltonian_*. */
int qed_new_model_generators(const char *name, int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep);

/* Hamiltonian<double> of one sector in the symmetry-adapted basis
 * (Hamiltonian_CSR over ED_mixed_basis: src_ed/Hamiltonian/Hamiltonian_CSR.hpp,
 * src_ed/ED_basis.cpp:185-385, src_ed/Operators/HS_one_body_operator.hpp:11-39),
 * built and kept on the device. dim is the basis dimension. */
typedef struct qed_mixed_hamiltonian qed_mixed_hamiltonian;
int qed_mixed_hamiltonian_create(int label, const char *sector, qed_mixed_hamiltonian **h, long *dim);
/* the basis: sorted representative states (spin up in bits 0-31) */
int qed_mixed_hamiltonian_states(qed_mixed_hamiltonian *h, uint64_t *states);
/* y += H x on host vectors of dim doubles (Hamiltonian::mult_add) */
int qed_mixed_hamiltonian_mult_add(qed_mixed_hamiltonian *h, const double *x, double *y);
/* y = H x on device vectors, enqueued on `stream` (a cudaStream_t; NULL: default) */
int qed_mixed_hamiltonian_apply_device(qed_mixed_hamiltonian *h, const double *x, double *y, void *stream);
/* lowest eigenvalue of the sector by Lanczos (LanczosEigenvalue,
 * src_ed/Hamiltonian/Lanczos.hpp:41-97; accur_lanczos, max_iter_lanczos, seed) */
int qed_mixed_hamiltonian_ground_state(qed_mixed_hamiltonian *h, double *energy, int *iterations);
/* the ground-state energy and vector (dim doubles, in the basis order of
 * qed_mixed_hamiltonian_states) by the two Lanczos passes (LanczosEigenvalue and
 * LanczosEigenvector, src_ed/Hamiltonian/Lanczos.hpp:41-143) */
int qed_mixed_hamiltonian_ground_state_vector(qed_mixed_hamiltonian *h, double *energy, double *psi);
/* number of stored off-diagonal entries */
int qed_mixed_hamiltonian_nnz(qed_mixed_hamiltonian *h, long *nnz);
int qed_mixed_hamiltonian_destroy(qed_mixed_hamiltonian *h);

/* symmetry_group::build (src_ed/symmetry_group.cpp:184-345): the group order g,
 * the character phases phi (g x g, units of 2 pi / g), the symmetric site
 * orbitals S (n_sites x n_sites row-major, real and imaginary parts; row k is
 * the k-th orbital, irreps in order) and the number of them in each irrep
 * (site_irrep_dim, g entries). Output pointers may be NULL; phi and
 * site_irrep_dim need room for 16 x 16 and 16 entries when g is not known. */
int qed_symmetry_group(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int *g, int *phi,
                       double *S_re, double *S_im, int *site_irrep_dim);

/* symmetry_group::Representative (src_ed/symmetry_group.cpp:231-262) of n basis
 * states (spin up in bits 0-31, spin down in bits 32-63) in irrep `irrep`: the
 * orbit's smallest state, the phase (units of pi / g) and the orbit length (0:
 * the projected state vanishes; rep and phase are then meaningless). */
int qed_symmetry_representatives(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int irrep,
                                 long n, const uint64_t *states, uint64_t *rep, int *phase, int *length);

/* ---- VCA surrogate network ---------------------------------------------------
 * No counterpart in the reference (its VCA, pyqcm/vca.py, evaluates the Potthoff
 * functional by ED at every point). A multilayer perceptron n_in -> W -> W -> W -> 1
 * (GELU) trained by Adam on Omega values this solver computes; it proposes the
 * starting point of the ED Newton-Raphson search. BF16 weights and activations in
 * the tensor-core products, FP32 accumulation, FP32 master weights and moments.
 * Parameter layout (FP32, qed_mlp_layout gives the 8 block offsets and the padded
 * input width k_in): W1 [W][k_in] (columns >= n_in zero), b1 [W], W2 [W][W], b2,
 * W3 [W][W], b3, w4 [W], b4 [1]. Errors: qed_mlp_last_error. */
int qed_mlp_create(int n_in, int width, unsigned long long seed, void **handle);
void qed_mlp_destroy(void *handle);
int qed_mlp_last_error(char *buf, int len);
int qed_mlp_num_params(void *handle, long *n);
int qed_mlp_layout(void *handle, long *offsets9);
int qed_mlp_get_params(void *handle, float *params);
int qed_mlp_set_params(void *handle, const float *params);
/* y[rows] for x[rows][n_in] (host arrays) */
int qed_mlp_forward(void *handle, int rows, const float *x, float *y);
/* gradients of the mean squared error over rows (a multiple of 16) into grads
 * (the parameter layout) and the loss */
int qed_mlp_gradients(void *handle, int rows, const float *x, const float *t, float *grads, float *loss);
/* `epochs` passes of Adam (lr; beta1 0.9, beta2 0.999, eps 1e-8) over shuffled
 * batches (a multiple of 16 rows); per epoch, the loss of its last batch */
int qed_mlp_train(void *handle, int rows, const float *x, const float *t, int epochs, int batch, float lr,
                  unsigned long long seed, float *epoch_loss);
/* The network's matrix product on its own: C[M][N] = A[M][K] B[N][K]^T with A, B
 * given as BF16 bit patterns (host arrays, K contiguous) and C in FP32, computed
 * by the tcgen05 kernel of the surrogate (fp32 accumulation in tensor memory).
 * K and N multiples of 16. No counterpart in the reference; it lets a test check
 * the tensor-core path on shapes the network does not use. */
int qed_mlp_tensor_product(int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C);

#ifdef __cplusplus
}
#endif
#endif /* QED_B200_H */
