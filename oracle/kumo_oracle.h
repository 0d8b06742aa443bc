/*
 * kumo_oracle: CPU restatement of chem-kumo's grid-block evaluator.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker of the CUDA path and
 * the timed CPU baseline; it is never linked into, loaded by or called from the
 * product library.  It restates, in plain C with the reference's operation
 * order where the reference source makes that order explicit, the functions
 * cited beside each declaration (paths inside the chem-kumo 2.1.0 sources).
 * Where the reference delegates to Eigen (matrix products, reductions, the
 * 3x3 eigensolver) this restatement sums left to right in index order.
 *
 * Parity pin: the restatement is checked against the reference's own golden
 * data (Gaussian cubegen densities of O2 and acrolein, Multiwfn ELF / RDG /
 * sign(lambda2)rho / ESP cubes of water, Boys-function known answers); see
 * tests/test_oracle_golden.py.
 *
 * Layouts: matrices are column-major like the reference's Eigen matrices:
 * element (row r, column c) of an R x C matrix is at [c * R + r].
 */
#ifndef KUMO_ORACLE_H
#define KUMO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ko_basis ko_basis;
typedef struct ko_esp ko_esp;

/* Density-derivative record of one point, as detail::DensityDerivatives
 * (include/chem/kumo/density.hpp:153-160); hess is 3x3 row-major. */
typedef struct {
    double value;
    double grad[3];
    double hess[9];
    double lap;
    double tau;
    double tau_axes[3];
} ko_dd;

typedef struct {
    int kind;          /* PropertyKind, include/chem/kumo/evaluator.hpp:109-153 */
    int component;     /* DensityComponent: Total 0, Alpha 1, Beta 2, Difference 3 */
    int channel;       /* SpinChannel: Alpha 0, Beta 1 */
    long orbital_index;/* one-based */
} ko_property;

typedef struct {
    const ko_basis* basis;
    const double* p_total;   /* n x n */
    const double* p_spin;    /* n x n */
    const double* c_alpha;   /* n x nmo_alpha, one MO per column */
    int nmo_alpha;
    const double* c_beta;    /* n x nmo_beta, NULL for restricted */
    int nmo_beta;
    int nalpha, nbeta;
    int ao_mo_eligible;
    int natoms;
    const double* atom_xyz;    /* 3 * natoms */
    const double* atom_charge; /* natoms */
} ko_molecule;

typedef struct {
    long block_size;            /* include/chem/kumo/evaluator.hpp:412 */
    int backend;                /* 0 AUTO, 1 AO_P, 2 AO_MO */
    double screening_threshold; /* include/chem/kumo/density.hpp:28 */
    double potential_tolerance; /* only 0 (exact) is restated */
} ko_options;

/* ---- basis preparation: src/basis.cpp:21-120, src/basis_math.cpp:9-66,
 *      src/basis_evaluator.cpp:49-202 ---- */
ko_basis* ko_basis_create(int nshell, const int* shell_types, const int* nprim,
                          const double* exps, const double* coefs, const double* p_coefs,
                          const double* shell_xyz, int declared_nbasis, char* err, int errlen);
void ko_basis_destroy(ko_basis* b);
int ko_basis_nao(const ko_basis* b);
int ko_basis_nblocks(const ko_basis* b);
/* l, nprim, offset, count, pure flag, cutoff radius squared of AO block i */
void ko_basis_block(const ko_basis* b, int i, int* l, int* nprim, int* offset, int* count,
                    int* pure, double* cutoff_r2);
/* Cartesian-to-pure matrix (2l+1) x ncart, column-major; src/basis_evaluator.cpp:157-175 */
void ko_pure_transform(int l, double* out);
double ko_primitive_norm(double alpha, int px, int py, int pz);

/* ---- AO kernels ---- */
/* evaluate_batch / evaluate_into_impl, src/basis_evaluator.cpp:413-488,665-678:
 * out is nao x b */
void ko_ao_values_batch(const ko_basis* b, const double* pts, int npts, double* out);
/* evaluate_derivatives_batch, src/basis_evaluator.cpp:512-643: out is
 * nao x (panels * npts), component c of point j in column c * npts + j */
void ko_ao_derivatives_batch(const ko_basis* b, const double* pts, int npts, int order, double* out);
/* significant_aos, src/ao_screening.hpp:35-50: keep[row] = 0/1 */
void ko_significant_aos(const double* ao, int rows, long cols, double threshold,
                        unsigned char* keep);

/* ---- density kernels (src/density.cpp) ---- */
/* density_derivatives_mo, src/density.cpp:235-351; out[c] (c = component) is
 * npts records or NULL when not requested */
int ko_density_derivatives_mo(const ko_molecule* m, const double* pts, long npts, long block,
                              int ao_order, double threshold, ko_dd* const out[4]);
/* density_derivatives_shared, src/density.cpp:150-229 */
int ko_density_derivatives_shared(const ko_molecule* m, const double* pts, long npts, long block,
                                  int ao_order, double threshold, ko_dd* const out[4]);
/* densities_blocked for one component, src/density.cpp:366-444 */
int ko_densities_blocked(const ko_molecule* m, const double* pts, long npts, long block,
                         double threshold, int component, double* out);
/* Molecule::orbitals, src/orbitals.cpp:66-102 (blocks of 128, values only) */
int ko_orbitals(const ko_molecule* m, const double* pts, long npts, int channel,
                const long* indices, int nidx, double* const* out);

/* ---- evaluator (src/evaluator.cpp, src/evaluation_plan.hpp,
 *      src/automatic_backend.hpp) ---- */
/* Grid: origin[3], steps[9] column-major (column = axis), counts[3]; or
 * explicit points (3 x npts) when origin is NULL.  outputs[p] holds
 * channels(kind) arrays of npts values, component-major. */
int ko_evaluate(const ko_molecule* m, const ko_options* opt, const double* origin,
                const double* steps, const int* counts, const double* points, long npoints,
                const ko_property* props, int nprops, double* const* outputs, int* backend_used,
                char* err, int errlen);
/* validate_orbital_backend, src/backend_selection.hpp:43-78; returns 1 if eligible */
int ko_validate_orbital_backend(int n, const double* total, const double* spin,
                                const double* alpha, int nmo_a, const double* beta, int nmo_b,
                                int nalpha, int nbeta, int unrestricted, double* errors4);
/* grid_point, src/grid_geometry.hpp:59-68 */
void ko_grid_points(const double* origin, const double* steps, const int* counts, long start,
                    long count, double* out);

/* ---- Boys function and electrostatic potential ---- */
/* boys_function, src/boys_function.cpp:47-76 */
int ko_boys(double t, int nvalues, double* values);
/* ElectrostaticPotential ctor, src/electrostatic_potential.cpp:117-229 */
ko_esp* ko_esp_create(const ko_basis* b, const double* p_total, int natoms, const double* xyz,
                      const double* charges);
void ko_esp_destroy(ko_esp* e);
long ko_esp_pair_count(const ko_esp* e);
/* Exact potential (tolerance 0), src/electrostatic_potential.cpp:231-360 */
void ko_esp_evaluate(const ko_esp* e, const double* pts, long npts, double* out);
void ko_esp_nuclear(const ko_esp* e, const double* pts, long npts, double* out);

/* OpenMP thread count used by the blocked loops (0 = runtime default). */
void ko_set_threads(int n);
int ko_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
