/*
 * kumo_b200.h: C ABI of the B200 grid evaluator for chem-kumo.
 *
 * Plain pointers and sizes only.  Every entry point returns a kumo_status
 * and, where it takes one, writes a one-line message into `err` (errlen
 * bytes, NUL-terminated).  Status codes map the exception types of the
 * chem-kumo C++ API: KUMO_INVALID_ARGUMENT = std::invalid_argument,
 * KUMO_OUT_OF_RANGE = std::out_of_range, KUMO_RUNTIME_ERROR =
 * std::runtime_error; device failures are KUMO_CUDA_ERROR and never abort.
 *
 * Reference interfaces are cited as path:line inside the chem-kumo 2.1.0
 * sources.  Layout conventions:
 *  - points: 3 x N, point j at points[3j .. 3j+2] (bohr), like the columns of
 *    the reference's Eigen::Matrix<double, 3, Dynamic>;
 *  - a grid: origin[3], steps[9] with steps[3a + r] = component r of the step
 *    vector of axis a, counts[3]; values in Field order (k fastest);
 *  - property outputs: channels(kind) arrays of N doubles, component-major
 *    (gradient x, y, z; Hessian xx, xy, xz, yy, yz, zz).
 */
#ifndef KUMO_B200_H
#define KUMO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KUMO_B200_ABI_VERSION 1

typedef enum {
    KUMO_OK = 0,
    KUMO_INVALID_ARGUMENT = 1,
    KUMO_OUT_OF_RANGE = 2,
    KUMO_RUNTIME_ERROR = 3,
    KUMO_CUDA_ERROR = 4,
    KUMO_OUT_OF_MEMORY = 5
} kumo_status;

/* Backend (include/chem/kumo/evaluator.hpp:403): 0 AUTO, 1 AO_P, 2 AO_MO. */
/* Precision: 0 FP64, 1 mixed (FP32 AO values, tensor-core contractions). */

/* One requested property (include/chem/kumo/evaluator.hpp:174-187): kind is
 * the PropertyKind value (evaluator.hpp:109-153), component the
 * DensityComponent (spin.hpp: Total 0, Alpha 1, Beta 2, Difference 3),
 * channel the SpinChannel (Alpha 0, Beta 1), orbital_index one-based. */
typedef struct {
    int kind;
    int component;
    int channel;
    long long orbital_index;
} kumo_property;

/* EvaluationOptions (include/chem/kumo/evaluator.hpp:406-441) plus the
 * arithmetic precision. */
typedef struct {
    long long block_size;       /* screening block, 1..65536 points (default 128) */
    int backend;
    double screening_threshold; /* default 1e-12 */
    double potential_tolerance; /* 0: exact electrostatic potential */
    int precision;
    double fukui_delta;         /* Gaussian width of the orbital-weighted Fukui weights (default 0.1 hartree) */
} kumo_options;

typedef struct {
    double origin[3];
    double steps[9];
    int counts[3];
} kumo_grid;

typedef struct {
    int natoms;
    int nbasis;
    int nalpha, nbeta;
    int nmo_alpha, nmo_beta;
    int unrestricted;
    int ao_mo_eligible;        /* ElectronicStructureInfo::ao_mo_eligible() */
    double check_errors[4];    /* total abs, total rel, spin abs, spin rel */
    int nblocks;               /* AO blocks after splitting SP shells */
    long long device_bytes;    /* HBM held by the resident copy (0 before first use) */
} kumo_molecule_info;

/* Opaque molecule: the host Molecule and its device-resident copy (AO
 * tables, density matrices, MO coefficients). */
typedef struct kumo_molecule kumo_molecule;

/* Fill *opt with the reference defaults (block 128, AUTO, 1e-12, 1e-8, FP64, Fukui delta 0.1). */
void kumo_default_options(kumo_options* opt);

/* Select the CUDA device used by the calls of this thread (one process per
 * GPU; no counterpart in the CPU-only reference). */
int kumo_set_device(int device, char* err, size_t errlen);

/* Load every kernel of this library on the current device now, once per
 * device (no counterpart in the CPU-only reference).  CUDA otherwise loads
 * each kernel at its first launch, and every host thread launching meanwhile
 * waits; latency-sensitive callers make this call before taking traffic
 * (kumo_server_create makes it).  kumo_registered_kernels returns how many
 * kernel instantiations the library lists (available without a GPU). */
int kumo_preload_kernels(char* err, size_t errlen);
int kumo_registered_kernels(void);

/* Molecule::from_fchk (include/chem/kumo/density.hpp:218; src/molecule.cpp:153-180). */
int kumo_molecule_from_fchk(const char* path, kumo_molecule** out, char* err, size_t errlen);

/* Molecule from in-memory FCHK records (the records read by
 * src/basis.cpp:21-48 and src/molecule.cpp:39-180): shell types, primitive
 * counts, shell-to-atom map (one-based), exponents, contraction and P(S=P)
 * coefficients (p_coefs may be NULL), shell coordinates; packed lower
 * triangles of the total and spin density matrices (spin may be NULL);
 * MO coefficients MO by MO (AO fastest; beta NULL for restricted). */
int kumo_molecule_from_arrays(int natoms, const int* atomic_numbers, const double* nuclear_charges,
                              const double* coordinates, int nshell, const int* shell_types,
                              const int* nprim, const int* shell_atom, const double* exponents,
                              const double* coefs, const double* p_coefs, const double* shell_xyz,
                              int nbasis, const double* packed_total, const double* packed_spin,
                              int nalpha, int nbeta, const double* alpha_mos, int nmo_alpha,
                              const double* beta_mos, int nmo_beta, kumo_molecule** out, char* err,
                              size_t errlen);

void kumo_molecule_destroy(kumo_molecule* m);

/* Molecule::atoms, electronic_structure_info, basis_size, occupied_count,
 * orbital_count (include/chem/kumo/density.hpp:221-256). */
int kumo_molecule_info_get(const kumo_molecule* m, kumo_molecule_info* info);
/* atomic numbers (natoms), nuclear charges (natoms), positions (3 natoms). */
int kumo_molecule_atoms(const kumo_molecule* m, int* z, double* charges, double* xyz);
/* Prepared AO block i (BasisEvaluator::PreparedBlock,
 * include/chem/kumo/basis_evaluator.hpp:118-131): l, nprim, AO offset, AO
 * count, pure flag and squared cutoff radius. */
int kumo_molecule_block(const kumo_molecule* m, int i, int* l, int* nprim, int* offset, int* count,
                        int* pure, double* cutoff_r2);

/* Evaluator::evaluate(const Grid&, const Request&)
 * (include/chem/kumo/evaluator.hpp:506; src/evaluator.cpp:804-809).
 * outputs[i] (host) receives property i; *backend_used = 1 AO_P or 2 AO_MO. */
int kumo_evaluate_grid(const kumo_molecule* m, const kumo_options* opt, const kumo_grid* grid,
                       const kumo_property* props, int nprops, double* const* outputs,
                       int* backend_used, char* err, size_t errlen);

/* Evaluator::evaluate(points, request) (include/chem/kumo/evaluator.hpp:516-518;
 * src/evaluator.cpp:821-826); points and outputs on the host. */
int kumo_evaluate_points(const kumo_molecule* m, const kumo_options* opt, const double* points,
                         long long npoints, const kumo_property* props, int nprops,
                         double* const* outputs, int* backend_used, char* err, size_t errlen);

/* Device-resident forms of the two calls above: outputs (and points) are
 * device pointers, work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns once it is queued. */
int kumo_evaluate_grid_device(const kumo_molecule* m, const kumo_options* opt, const kumo_grid* grid,
                              const kumo_property* props, int nprops, double* const* outputs,
                              void* stream, int* backend_used, char* err, size_t errlen);
int kumo_evaluate_points_device(const kumo_molecule* m, const kumo_options* opt,
                                const double* device_points, long long npoints,
                                const kumo_property* props, int nprops, double* const* outputs,
                                void* stream, int* backend_used, char* err, size_t errlen);

/* No counterpart in the reference.  Density properties at device points,
 * FP64 AO-MO path, without allocating any device memory: for hosts that
 * cannot let a library call cudaMalloc (a serving process that budgets every
 * byte of HBM itself, an application whose memory manager owns the device,
 * or code that must not risk cudaMalloc blocking until the device is idle).
 * The AO scratch is a fixed 64 MiB array that the library reserves in every
 * GPU that loads it, until exit.  The molecule's device copy must already
 * exist (any earlier evaluation of it on this device makes it); points and
 * outputs are device memory supplied by the caller, the work is queued on
 * `stream`.  The first call on each device looks up the array's address;
 * make it before any stream capture.  All calls share the array, so calls
 * whose work overlaps on the GPU race: serialize them.  A molecule whose
 * scratch for one 128-point block exceeds the array is rejected with
 * KUMO_INVALID_ARGUMENT.  opt: block_size 1..128, backend AUTO or AO_MO,
 * precision FP64 (NULL for the defaults); every outputs[i] must be non-null.
 * The queued kernels read the molecule's device copy: do not evaluate the same
 * molecule on another device (which replaces that copy) or destroy it while
 * they may still run. */
int kumo_evaluate_points_noalloc(const kumo_molecule* m, const kumo_options* opt,
                                 const double* device_points, long long npoints,
                                 const kumo_property* props, int nprops, double* const* outputs,
                                 void* stream, char* err, size_t errlen);

/* BasisEvaluator::evaluate_derivatives_batch / evaluate_batch
 * (include/chem/kumo/basis_evaluator.hpp:101-115; src/basis_evaluator.cpp:512-678)
 * on the device: order 0 (values), 1 or 2; out (host) is nao x (panels*npts)
 * column-major, component c of point j in column c*npts + j.  npts <= 128. */
int kumo_ao_panels(const kumo_molecule* m, const double* points, int npts, int order, int precision,
                   double* out, char* err, size_t errlen);

/* Screening masks of significant_aos (src/ao_screening.hpp:35-50) for the
 * blocks of `block_size` points of a grid: mask (host) is nblocks x nao bytes,
 * 1 where the AO is kept.  ao_order selects the panels (0, 1 or 2). */
int kumo_screening_masks(const kumo_molecule* m, const kumo_grid* grid, long long block_size,
                         int ao_order, double threshold, unsigned char* mask, char* err,
                         size_t errlen);

/* detail::boys_function (src/boys_function.cpp:47-76) on the device:
 * out[i * nvalues + m] = F_m(t[i]), nvalues <= 33 (host arrays). */
int kumo_boys(const double* t, long long n, int nvalues, double* out, char* err, size_t errlen);

/* Number of primitive pairs of the electrostatic potential
 * (ElectrostaticPotential::primitive_pair_count, src/electrostatic_potential.hpp:61). */
int kumo_esp_pair_count(const kumo_molecule* m, long long* count, char* err, size_t errlen);

/* Primitive pairs the device evaluates for potential_tolerance `tolerance`
 * (the role of ElectrostaticPotential::far_field_plan,
 * src/electrostatic_potential.cpp:501-521): all of them for 0; otherwise those
 * left after dropping the pairs whose bounds (|contribution| at any point)
 * sum to at most tolerance / 2. */
int kumo_esp_pairs_evaluated(const kumo_molecule* m, double tolerance, long long* count, char* err, size_t errlen);

/* Field::write_cube / write_orbital_cube (include/chem/kumo/density.hpp:120-128;
 * src/cube.cpp:70-111); orbital_index 0 writes a density Cube. */
int kumo_write_cube(const char* path, const char* comment, const kumo_grid* grid, int natoms,
                    const int* atomic_numbers, const double* charges, const double* xyz,
                    const double* values, long long orbital_index, char* err, size_t errlen);

/* No counterpart in the reference.  The mixed form's tile-shape autotuner:
 * the shapes timed so far, one line per key (molecule, backend, panels,
 * exact rows, grid step lengths) with the candidates fastest first as
 * "AxBxC:time".  Copies at most len - 1 bytes and a NUL; returns the length
 * of the whole report. */
long long kumo_tile_tuning_report(char* buf, size_t len);

/* read_cube (include/chem/kumo/cube.hpp:32 of chem-kumo; src/cube.cpp:114-212):
 * a scalar Cube file, plain or gzip, into a handle; angstrom headers are
 * converted to bohr.  kumo_cube_info gives the atom count, the grid (bohr)
 * and whether the header was in angstrom; kumo_cube_data copies the atoms
 * (z, charges, xyz as natoms x 3), the values (Field order) and the two
 * comment lines (truncated to their buffers, NUL-terminated); any output
 * pointer may be NULL. */
typedef struct kumo_cube kumo_cube;
int kumo_read_cube(const char* path, kumo_cube** out, char* err, size_t errlen);
int kumo_cube_info(const kumo_cube* c, long long* natoms, kumo_grid* grid, int* angstrom);
int kumo_cube_data(const kumo_cube* c, int* atomic_numbers, double* charges, double* xyz, double* values,
                   char* first_comment, size_t first_len, char* second_comment, size_t second_len);
void kumo_cube_destroy(kumo_cube* c);
/* write_cube(CubeData) (include/chem/kumo/cube.hpp:38; src/cube.cpp:215-251):
 * 13 significant digits, the given comment lines and length unit (angstrom
 * != 0: the header in angstrom, negative counts), so that kumo_read_cube
 * reproduces the field to 13 digits.  Grid, atoms and values in bohr. */
int kumo_write_cube_data(const char* path, const char* first_comment, const char* second_comment, int angstrom,
                         const kumo_grid* grid, long long natoms, const int* atomic_numbers,
                         const double* charges, const double* xyz, const double* values, char* err,
                         size_t errlen);

/* Grid::around / line / plane (include/chem/kumo/density.hpp:72-91). */
int kumo_grid_around(const kumo_molecule* m, double margin, double spacing, kumo_grid* out,
                     char* err, size_t errlen);

/* Kernel timing of the evaluation waves (no counterpart in the reference,
 * whose benchmarks time whole calls): when enabled, every launch of the
 * device kernels is bracketed by CUDA events on its stream and the kept AO
 * rows of every screening block are summed on the device. */
typedef struct {
    char name[32];
    int launches;
    double ms;        /* summed event time */
    double kept_rows; /* sum over blocks of the kept AO rows */
    double units;     /* blocks (AO build, contractions) or point-pair interactions (ESP) */
    double flops;     /* algorithmic FLOPs of the contractions */
    double bytes;
} kumo_profile_entry;

void kumo_profile_enable(int on);
void kumo_profile_reset(void);
/* Synchronizes and returns the number of entries written (<= max_entries). */
int kumo_profile_read(kumo_profile_entry* out, int max_entries);

/* ---- Serving loop (new: chem-kumo has no serving counterpart) -----------
 * A server queues evaluation requests of any molecules and sizes, admits them
 * in arrival order while their device-memory footprint fits an HBM budget and
 * one of max_active slots (CUDA streams) is free, and runs the admitted ones
 * concurrently so that their kernels overlap on the GPU; requests of at most
 * graph_points points replay CUDA graphs captured per (molecule, options,
 * properties, point bucket).  Results go to the caller's host arrays (which,
 * like the molecule, must stay valid until the request is done); latency runs
 * from submit until the results are in those arrays.  Zero option fields take
 * the defaults: budget 150 GB capped at 90% of free memory, 8 slots, 65536
 * graph points (negative: no graphs), 1 GiB AO scratch per request. */
typedef struct kumo_server kumo_server;

typedef struct {
    int device;
    double hbm_budget_bytes;
    int max_active;
    long long graph_points;
    double request_scratch_bytes;
    double staging_bytes; /* page-locked staging arena (0: 2 GiB; negative: none) */
} kumo_server_options;

typedef struct {
    long long submitted, completed, failed, points;
    double p50_ms, p99_ms, mean_ms, max_ms;
    double busy_s;        /* first submit to last completion */
    double points_per_s;  /* completed points / busy_s */
    long long graph_captures, graph_replays, direct_runs;
    double peak_bytes, budget_bytes;
    double launch_s;  /* scheduler host time issuing requests */
    double copy_s;    /* completion-thread time copying results */
    double queue_ms;  /* mean submit-to-admission time */
} kumo_server_stats;

int kumo_server_create(const kumo_server_options* opt, kumo_server** out, char* err, size_t errlen);
/* Waits for every submitted request, then frees the server. */
int kumo_server_destroy(kumo_server* server);
int kumo_server_submit_grid(kumo_server* server, const kumo_molecule* m, const kumo_options* opt,
                            const kumo_grid* grid, const kumo_property* props, int nprops,
                            double* const* outputs, unsigned long long* ticket, char* err, size_t errlen);
int kumo_server_submit_points(kumo_server* server, const kumo_molecule* m, const kumo_options* opt,
                              const double* points, long long npoints, const kumo_property* props, int nprops,
                              double* const* outputs, unsigned long long* ticket, char* err, size_t errlen);
/* done = 1 once the ticket's results are in the caller's arrays (within timeout_s);
 * a failed request returns its error status and message. */
int kumo_server_wait(kumo_server* server, unsigned long long ticket, double timeout_s, int* done, char* err,
                     size_t errlen);
int kumo_server_drain(kumo_server* server, char* err, size_t errlen);
int kumo_server_stats_get(kumo_server* server, kumo_server_stats* out, char* err, size_t errlen);
int kumo_server_reset_stats(kumo_server* server, char* err, size_t errlen);

/* ---- Molecular surfaces (include/chem/kumo/surface.hpp) ------------------
 * A kumo_surface holds a closed triangle mesh (vertices in bohr; triangles
 * counter-clockwise seen from outside) and, per mapped field, one value per
 * vertex with its surface statistics. */
typedef struct kumo_surface kumo_surface;

/* SurfaceStatistics (include/chem/kumo/surface.hpp:37-77); the local minima
 * and maxima (vertex indices, sorted) are copied separately. */
typedef struct {
    double area, positive_area, negative_area, nonpolar_area;
    double minimum, maximum;
    long long minimum_vertex, maximum_vertex;
    double average, positive_average, negative_average;
    double positive_variance, negative_variance, total_variance;
    double balance, charge_separation, polarity_index;
    long long n_local_minima, n_local_maxima;
} kumo_surface_stats;

/* density_isosurface (include/chem/kumo/surface.hpp:101-116; src/surface.cpp:329-535). */
int kumo_density_isosurface(const kumo_molecule* m, double isovalue, double spacing, kumo_surface** out,
                            char* err, size_t errlen);
/* electrostatic_potential_surface (surface.hpp:118-133; src/surface.cpp:586-631): field 0
 * is the potential (exact; any tolerance >= 0 is met). */
int kumo_potential_surface(const kumo_molecule* m, double isovalue, double spacing, double tolerance,
                           kumo_surface** out, char* err, size_t errlen);
/* local_ionization_energy_surface (surface.hpp:157-165; src/surface.cpp:568-584): field 0. */
int kumo_ionization_energy_surface(const kumo_molecule* m, double isovalue, double spacing, kumo_surface** out,
                                   char* err, size_t errlen);
/* map_on_density_isosurface (surface.hpp:167-192; src/surface.cpp:633-670): one field per
 * distinct property, in request order; *backend_used as kumo_evaluate_*. */
int kumo_map_on_density_isosurface(const kumo_molecule* m, const kumo_options* opt, const kumo_property* props,
                                   int nprops, double isovalue, double spacing, kumo_surface** out,
                                   int* backend_used, char* err, size_t errlen);
/* average_local_ionization_energy at points (surface.hpp:135-155; src/surface.cpp:537-566). */
int kumo_average_local_ionization_energy(const kumo_molecule* m, const double* points, long long npoints,
                                         double* out, char* err, size_t errlen);

/* f and its gradient at n points (3 x n, bohr): values[n], gradients[3n]. */
typedef void (*kumo_scalar_fn)(const double* points, long long n, double* values, double* gradients, void* user);
/* detail::extract_isosurface (src/isosurface.hpp; src/surface.cpp:296-320): the
 * isosurface f = isovalue of host samples on a grid, vertices placed with fn. */
int kumo_extract_isosurface(const kumo_grid* grid, const double* samples, double isovalue, kumo_scalar_fn fn,
                            void* user, kumo_surface** out, char* err, size_t errlen);

void kumo_surface_info(const kumo_surface* s, long long* nvertices, long long* ntriangles, int* nfields);
/* vertices: 3 x nvertices; triangles: 3 x ntriangles; cells (may be NULL): the
 * grid indices of the lower end of each vertex's edge, 3 x nvertices. */
void kumo_surface_mesh(const kumo_surface* s, double* vertices, long long* triangles, int* cells);
/* Field `index`: values (nvertices) and statistics; minima / maxima receive up
 * to cap_min / cap_max vertex indices (either may be NULL). */
int kumo_surface_field(const kumo_surface* s, int index, double* values, kumo_surface_stats* stats,
                       long long* minima, long long cap_min, long long* maxima, long long cap_max, char* err,
                       size_t errlen);
void kumo_surface_destroy(kumo_surface* s);

/* surface_statistics (surface.hpp:79-86; src/surface.cpp:417-531) of vertex values on a mesh. */
int kumo_surface_statistics(const double* vertices, long long nvertices, const long long* triangles,
                            long long ntriangles, const double* values, double polar_threshold,
                            kumo_surface_stats* out, long long* minima, long long cap_min, long long* maxima,
                            long long cap_max, char* err, size_t errlen);
/* write_ply (surface.hpp:194-208; src/surface.cpp:672-720). */
int kumo_write_ply(const char* path, const double* vertices, long long nvertices, const long long* triangles,
                   long long ntriangles, const char* const* names, const double* const* values, int nfields,
                   const char* const* comments, int ncomments, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif
