/*
 * cubismnova_b200.h -- C ABI of the B200-native CubismNova lab/stencil path.
 *
 * The reference (CubismNova 0.6.0) is a header-only C++ template library with
 * no FFI of its own.  The entry points below are the seams a replacement slots
 * behind; each one names the reference interface it replaces (file:line
 * within the CubismNova source tree).
 *
 * Conventions
 *   - All functions return cn_status (0 == CN_OK); no C++ exception crosses
 *     this boundary.  cn_last_error_string() holds the message of the last
 *     failure on the calling thread, using the reference's own strings where
 *     the reference throws.
 *   - The library owns device memory of a grid; callers own host buffers.
 *   - "stream" is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Every call with a stream argument is stream-ordered and
 *     returns without waiting for the device unless stated otherwise.
 *   - Grid data layout on the device is the reference layout
 *     (Grid/Cartesian.h:490-529, Grid/BlockFieldAssembler.h:189-194):
 *     component-major, then block-major in x-fastest block order, each block
 *     block_cells[0]*block_cells[1]*block_cells[2] cells x-fastest, blocks
 *     block_stride elements apart (cells*sizeof rounded up to 32 bytes).
 *     A host array in the reference's SoA order uploads with one copy.
 *   - Fused stencil operators take cell-centred grids; node and face grids
 *     (cn_grid_create_entity) work with labs, BCs, the lab fill and IO.
 */
#ifndef CUBISMNOVA_B200_H
#define CUBISMNOVA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CN_ABI_VERSION 1

typedef enum cn_status {
    CN_OK = 0,
    CN_ERR_INVALID_ARGUMENT = 1,
    CN_ERR_STENCIL_BEGIN = 2,    /* "Stencil: begin_ must be <= 0" (Core/Stencil.h:101-102) */
    CN_ERR_STENCIL_END = 3,      /* "Stencil: end_ must be > 0" (Core/Stencil.h:104-105) */
    CN_ERR_STENCIL_COMPONENT = 4,/* a single component violates begin<=0 / end>0 */
    CN_ERR_NOT_ALLOCATED = 5,    /* "FieldLab: can not load lab data when not allocated first" (Block/FieldLab.h:189-190) */
    CN_ERR_NO_FIELD = 6,         /* "FieldLab: no field loaded" (Block/FieldLab.h:417-419) */
    CN_ERR_SIZE_MISMATCH = 7,    /* "Cartesian: Can not assign two grids of unequal size." (Grid/Cartesian.h:162-164) */
    CN_ERR_STENCIL_TOO_WIDE = 8, /* ghost width larger than the block in some dimension */
    CN_ERR_CUDA = 9,             /* a CUDA runtime call failed */
    CN_ERR_OUT_OF_MEMORY = 10,
    CN_ERR_DEVICE = 11,          /* a kernel reported an error word */
    CN_ERR_UNSUPPORTED = 12,
    CN_ERR_TOO_MANY_BC = 13,
    CN_ERR_FILE = 14             /* a file could not be opened, read or written, or is not a readable HDF5 file */
} cn_status;

typedef enum cn_dtype { CN_FLOAT32 = 0, CN_FLOAT64 = 1, CN_INT32 = 2 } cn_dtype;

/* Cubism::EntityType (Common.h) of a grid's values: cell centres, nodes
 * (cells + 1 per block and direction), or the faces normal to x, y or z
 * (cells + 1 along that direction).  A reference FaceContainer grid is three
 * face grids, one per direction. */
typedef enum cn_entity {
    CN_ENTITY_CELL = 0,
    CN_ENTITY_NODE = 1,
    CN_ENTITY_FACE_X = 2,
    CN_ENTITY_FACE_Y = 3,
    CN_ENTITY_FACE_Z = 4
} cn_entity;

/* BC::Base (periodic no-op) / BC::Dirichlet / BC::Absorbing / BC::Symmetry
 * (BC/Base.h:39-79, BC/Dirichlet.h:38, BC/Absorbing.h:35, BC/Symmetry.h:43) */
typedef enum cn_bc_kind {
    CN_BC_BASE = 0,
    CN_BC_DIRICHLET = 1,
    CN_BC_ABSORBING = 2,
    CN_BC_SYMMETRY = 3
} cn_bc_kind;

/* Core::Stencil(begin, end, tensorial) (Core/Stencil.h:44-67): begin <= 0
 * inclusive, end > 0 exclusive; tensorial labs include edge/corner ghosts. */
typedef struct cn_stencil {
    int begin[3];
    int end[3];
    int tensorial;
} cn_stencil;

typedef struct cn_grid cn_grid;

/* ------------------------------------------------------- device memory */
/* Plain device buffers for callers without the CUDA runtime headers (the C++
 * facade's lab storage).  cn_memcpy copies in any direction (stream NULL:
 * returns when done). */
cn_status cn_device_alloc(size_t bytes, void **ptr);
cn_status cn_device_free(void *ptr);
cn_status cn_memcpy(void *dst, const void *src, size_t bytes, void *stream);

/* ---------------------------------------------------------------- errors */
const char *cn_status_string(cn_status s);
/* Message of the last failed call on this thread ("" if none). */
const char *cn_last_error_string(void);
int cn_abi_version(void);

/* Validates a stencil exactly like Core::Stencil::check_
 * (Core/Stencil.h:99-107), then rejects single-component violations. */
cn_status cn_stencil_check(const cn_stencil *s);

/* ------------------------------------------------------------------ grid */
/* Grid::Cartesian(nblocks, block_cells, begin, end) (Grid/Cartesian.h:132-143)
 * with ncomp scalar components (rank-0: 1, rank-1 vector: 3, Euler state: 5).
 * Allocates the device storage on the current CUDA device. */
cn_status cn_grid_create(const int nblocks[3], const int block_cells[3], int ncomp,
                         cn_dtype dtype, const double begin[3], const double end[3],
                         cn_grid **out);
/* The same for node and face entities (Grid/Cartesian.h:490-513): the block
 * extent is block_cells (+1 for nodes, +1 along the face direction); every
 * lab, BC and stencil entry point works on that extent (FieldLab.h:104-224
 * with the entity's index range), the cell size h stays (end-begin)/cells. */
cn_status cn_grid_create_entity(const int nblocks[3], const int block_cells[3], int ncomp, cn_dtype dtype,
                                cn_entity entity, const double begin[3], const double end[3], cn_grid **out);
/* Entity type and block cells of a grid (its block extent is cn_grid_shape's). */
cn_status cn_grid_entity(const cn_grid *g, int *entity, int block_cells[3]);
cn_status cn_grid_destroy(cn_grid *g);
/* Layout in elements: block stride, component stride; total bytes. */
cn_status cn_grid_layout(const cn_grid *g, int64_t *block_stride, int64_t *comp_stride,
                         size_t *total_bytes);
/* nblocks[3], block_cells[3], ncomp, dtype of a grid (Grid/Cartesian.h:240-256). */
cn_status cn_grid_shape(const cn_grid *g, int info[8]);
/* Mesh::StructuredUniform cell size h = (end-begin)/cells
 * (Mesh/StructuredUniform.h:61, :333-336). */
cn_status cn_grid_cell_size(const cn_grid *g, double h[3]);
/* Device error word of a grid.  A kernel that reads the grid and gives up a
 * bounded wait (a TMA copy or tensor-core pipeline that did not complete)
 * records a nonzero word instead of hanging (1: a wait ran out, 2: a table
 * entry out of range, 3: unusable launch configuration) and skips its
 * results.  Waits for the device; clear != 0 resets the word.  The calls that
 * synchronise anyway (cn_euler_rk3_stage with sums, the no-allocation stage,
 * cn_mg_solve) return CN_ERR_DEVICE when it is set. */
cn_status cn_grid_device_error(cn_grid *g, int *word, int clear);
/* Test hook of that path: one CTA polls `polls` times (1..2^20) an mbarrier
 * that nothing completes, then records 1 in g's error word.  Stream-ordered;
 * no fault, the context stays usable. */
cn_status cn_debug_wait_timeout(cn_grid *g, int polls, void *stream);
/* Device pointer of one component (component-major SoA). */
cn_status cn_grid_data(cn_grid *g, int comp, void **device_ptr);
/* Host <-> device copy of one component, reference SoA order; nbytes must be
 * comp_stride*sizeof(dtype).  Blocking unless the host memory is pinned. */
cn_status cn_grid_upload(cn_grid *g, int comp, const void *host, size_t nbytes, void *stream);
cn_status cn_grid_download(const cn_grid *g, int comp, void *host, size_t nbytes, void *stream);
/* Cartesian::operator= (Grid/Cartesian.h:160-169): copy all block data. */
cn_status cn_grid_copy(cn_grid *dst, const cn_grid *src, void *stream);

/* -------------------------------------------------------------------- IO */
/* Field2AOS over every block of a grid, as CartesianWriteHDF's block loop
 * (IO/CartesianHDF.h:76-80; IO/FieldAOS.h:37-57 scalar, :79-101 tensor,
 * :136-141 face field of one direction = that direction's face grid here).
 * The file range [span_begin, span_end) is a box of global entity indices
 * (the HDF dataset, x fastest); for every point p of it inside the grid,
 *   d_buf[c + ncomp * flat(p - span_begin)] = (file type) component comp0 + c at p,
 * c < ncomp <= 16.  Points of the range outside the grid are not written.
 * d_buf is device (or managed / pinned host) memory of span volume * ncomp
 * elements of file_dtype; other host memory is rejected (CN_ERR_INVALID_ARGUMENT).
 * Conversions follow C++ (double -> float rounds to nearest); a
 * floating-point grid cannot be written as int32 (CN_ERR_UNSUPPORTED).
 * Stream-ordered; no allocation. */
cn_status cn_grid_to_aos(cn_grid *g, int comp0, int ncomp, const int span_begin[3], const int span_end[3],
                         cn_dtype file_dtype, void *d_buf, void *stream);
/* AOS2Field over every block (IO/FieldAOS.h:59-77, :103-124; the block loop
 * of CartesianReadHDF, IO/CartesianHDF.h:182-186): component comp0 + c at p
 *   = (grid type) d_buf[c + ncomp * flat(p - span_begin)]
 * for every point p of the range inside the grid; other grid points keep
 * their values.  A floating-point file cannot be read into an int32 grid
 * (CN_ERR_UNSUPPORTED). */
cn_status cn_grid_from_aos(cn_grid *g, int comp0, int ncomp, const int span_begin[3], const int span_end[3],
                           cn_dtype file_dtype, const void *d_buf, void *stream);

/* ------------------------------------------------------- HDF5 / XDMF files */
/* IO::CartesianWriteHDF of a grid (IO/CartesianHDF.h:42-96 with
 * src/IO/HDFDriver.cpp:25-111): the file range [begin, end) of components
 * [comp0, comp0 + ncomp) (ncomp < 0: all from comp0) gathered on the device
 * (cn_grid_to_aos), written as dataset "data" of dims (z, y, x, ncomp) and
 * type file_dtype into `fname.h5`; with create_xdmf, the reference's
 * message "CartesianWriteHDF: Allocating %.1f MB file buffer (fname)" on
 * stdout and, for cell and node data, the XDMF wrapper `fname.xmf`
 * (IO/XDMFDriver.h:31-160, Format="HDF", "./basename.h5:/data").
 * The HDF5 file is written without libhdf5, in the format libhdf5 writes
 * with its default bounds (superblock 0, v1 object headers); the data is
 * contiguous.  Synchronises the stream. */
cn_status cn_grid_write_hdf(cn_grid *g, const char *fname, const char *aname, int comp0, int ncomp,
                            const int begin[3], const int end[3], cn_dtype file_dtype, double time,
                            int create_xdmf, void *stream);
/* IO::CartesianReadHDF (IO/CartesianHDF.h:147-192 with
 * src/IO/HDFDriver.cpp:113-165): reads the hyperslab [0, count) of dataset
 * "data" in `fname.h5` (count = the range's (z, y, x) extent and ncomp,
 * values converted to file_dtype) into the range of the grid
 * (cn_grid_from_aos).  A missing file: CN_ERR_FILE with the reference's
 * message "CartesianReadHDF: File 'fname' does not exist".  Synchronises
 * the stream. */
cn_status cn_grid_read_hdf(cn_grid *g, const char *fname, int comp0, int ncomp, const int begin[3],
                           const int end[3], cn_dtype file_dtype, void *stream);
/* Host-side HDF5 files of one dataset (no GPU needed).
 * cn_h5_write: `path` with dataset `dataset` (root group) of `rank` dims,
 * row-major values of dtype from host_buf; chunked != 0 stores it as one
 * chunk (the reference's H5Pset_chunk(dims) layout, < 4 GiB), else
 * contiguous.
 * cn_h5_query: rank, dims and type of a dataset in the root group.
 * cn_h5_read: the hyperslab [0, count) of a dataset into host_buf (row-major,
 * dtype; file values converted: FP64 <-> FP32, integers -> any).  Reads files
 * of superblock version 0 or 1 (after a user block), old-style groups, v1
 * object headers and compact, contiguous or chunked (unfiltered) layouts. */
cn_status cn_h5_write(const char *path, const char *dataset, int rank, const long long *dims, cn_dtype dtype,
                      const void *host_buf, int chunked);
cn_status cn_h5_query(const char *path, const char *dataset, int *rank, long long dims[32], cn_dtype *dtype);
cn_status cn_h5_read(const char *path, const char *dataset, int rank, const long long *count, cn_dtype dtype,
                     void *host_buf);
/* The XDMF wrapper (IO/XDMFDriver.h:31-160) `fname.xmf` of the file range
 * [begin, end) of cell or node data on the uniform mesh with origin and
 * spacing h: format 0 refers to "./basename.h5:/data" (Format="HDF"),
 * format 1 to the raw little-endian file "./basename.bin" (Format="Binary"). */
cn_status cn_xdmf_write(const char *fname, const char *aname, cn_entity entity, const int begin[3],
                        const int end[3], const double origin[3], const double h[3], int ncomp,
                        cn_dtype file_dtype, double time, int format);

/* -------------------------------------------------------------------- BC */
/* field.getBC().push_back(new BC::Kind(dir, side, value))
 * (Block/Field.h:437-442) for block `block` (flat x-fastest index) of
 * component comp.  value = Dirichlet value or Symmetry sign; ignored
 * otherwise.  Order matters exactly as in the reference vector. */
cn_status cn_bc_push(cn_grid *g, int comp, int block, int dir, int side, cn_bc_kind kind,
                     double value);
/* Push the same BC to every block touching domain face (dir, side); the
 * usual way the reference's drivers attach BCs to a Cartesian grid. */
cn_status cn_bc_push_boundary(cn_grid *g, int comp, int dir, int side, cn_bc_kind kind,
                              double value);
/* Clear the BC vector of one block (block >= 0) or of all blocks (-1). */
cn_status cn_bc_clear(cn_grid *g, int comp, int block);
cn_status cn_bc_count(const cn_grid *g, int comp, int block, int *count);
/* Upload the BC tables now (otherwise done by the next kernel call); call it
 * before capturing kernels of this grid into a CUDA graph. */
cn_status cn_bc_sync(cn_grid *g, void *stream);

/* ------------------------------------------------------------------- lab */
/* Extent of the dense active lab range of one block for stencil s:
 * block_cells - begin + end - 1 (Block/FieldLab.h:199-202). */
cn_status cn_lab_extent(const cn_grid *g, const cn_stencil *s, int extent[3]);
/* Cartesian::loadLab / FieldLab::loadData (Grid/Cartesian.h:412-427,
 * Block/FieldLab.h:180-224) for blocks [block_begin, block_begin+count):
 * lab i is written to d_labs + i*prod(extent) elements, x fastest, lab cell
 * q (q_d in [begin_d, block_cells_d+end_d-1)) at offset
 * (q0-b0) + E0*((q1-b1) + E1*(q2-b2)).  Cells the reference leaves undefined
 * (corners of a non-tensorial lab, a skipped neighbour no valid BC covers)
 * are not written.  apply_bc = 0 skips the BCs (loadData(..., false)). */
cn_status cn_lab_fill(cn_grid *g, int comp, const cn_stencil *s, int block_begin,
                      int block_count, int apply_bc, void *d_labs, void *stream);

/* ------------------------------------------------------- fused stencils */
/* Each call fills the lab of every block (stencil (-1,2) non-tensorial, BCs
 * of the input component applied) and applies the stencil in the same
 * kernel, writing the output grid (same geometry and dtype, FLOAT64).
 *
 * 7-point Laplacian, grouping of Kernel/Laplacian/Laplacian.cpp:123-130:
 *   out = ihx2*((u[+x] - 2u) + u[-x]) + ihy2*(...) + ihz2*(...), no FMA. */
cn_status cn_laplacian(cn_grid *u, int comp, cn_grid *out, int out_comp, void *stream);
/* Central gradient, out_comp..out_comp+2 = 0.5*((u[+d]-u[-d]) * ih_d)
 * (Kernel/Divergence/nova/nova.cpp:113-126 per-direction terms), no FMA. */
cn_status cn_gradient(cn_grid *u, int comp, cn_grid *out, int out_comp, void *stream);
/* Laplacian and gradient from one lab load (one kernel). */
cn_status cn_lap_grad(cn_grid *u, int comp, cn_grid *lap, int lap_comp, cn_grid *grad,
                      int grad_comp, void *stream);
/* Divergence of components comp..comp+2 of v (nova.cpp:113-126):
 *   out = 0.5*((((v0[+x]-v0[-x])*ihx) + ((v1[+y]-v1[-y])*ihy)) + ((v2[+z]-v2[-z])*ihz)). */
cn_status cn_divergence(cn_grid *v, int comp, cn_grid *out, int out_comp, void *stream);

/* The kernel ABI of the reference's ISPC benchmark
 * (test/sandbox/Benchmarks/ISPC/BaseBenchmark.h:27-37) on DEVICE pointers:
 * dst = fac*(sum of 6 neighbours - 6*src), fac = 1/(factor*factor),
 * summation order of ISPC/CFD_2ndOrder/DDX/ddxGold.cpp:9-33, no FMA.
 * src points at the first inner element of a pitched lab.  Runs on the
 * legacy default stream and returns after launch. */
void cn_ddx_f64(int Nx, int Ny, int Nz, const double *src, int x_pitch_src, int xy_pitch_src,
                double *dst, int x_pitch_dst, int xy_pitch_dst, double factor);
void cn_ddx_f32(int Nx, int Ny, int Nz, const float *src, int x_pitch_src, int xy_pitch_src,
                float *dst, int x_pitch_dst, int xy_pitch_dst, float factor);
cn_status cn_ddx_async(cn_dtype dtype, int Nx, int Ny, int Nz, const void *src, int x_pitch_src,
                       int xy_pitch_src, void *dst, int x_pitch_dst, int xy_pitch_dst,
                       double factor, void *stream);

/* ------------------------------------------------- compressible Euler */
/* The reference promises WENO reconstruction operators (README.rst:28-31)
 * without code; these entry points implement the published method on the
 * lab of stencil (-3,4) non-tensorial, per-component BC vectors applied.
 * State: 5 components (rho, rho*u, rho*v, rho*w, E) of one grid, gamma-law
 * gas; WENO5-JS (eps 1e-6, linear weights 1/10, 6/10, 3/10) on primitive
 * variables, Rusanov flux, RHS = -sum_d (F_{i+1/2} - F_{i-1/2}) / h_d.
 * Block cells must be multiples of 8; FLOAT64 or FLOAT32 grids. */
cn_status cn_euler_rhs(cn_grid *U, int comp0, double gamma, cn_grid *rhs, int rhs_comp0,
                       void *stream);
/* One SSP-RK3 stage (Shu & Osher), BCs taken from bcsrc's BC vectors:
 *   stage 1: out = Us + dt L(Us)
 *   stage 2: out = 3/4 Un + 1/4 (Us + dt L(Us))
 *   stage 3: out = 1/3 Un + 2/3 (Us + dt L(Us))    (out may alias Un)
 * If sums_out is not NULL the FP64 sums of the 5 outputs times the cell
 * volume are returned (the call then waits for the stream). */
cn_status cn_euler_rk3_stage(cn_grid *bcsrc, cn_grid *Us, cn_grid *Un, cn_grid *out, int stage,
                             double dt, double gamma, double *sums_out, void *stream);
/* cn_euler_rk3_stage with sums_out required and no device allocation: the
 * per-tile partials live in a fixed device array of the library (no
 * counterpart in the reference).  For callers that must not allocate during a
 * run (a fixed device-memory budget owned by another allocator, no
 * cudaMalloc/cudaFree synchronisation mid-run).  Like cn_euler_rk3_stage with
 * sums it copies the sums to the host and waits for the stream.  Limit: at
 * most 32768 8^3 tiles (16.8M cells), else CN_ERR_UNSUPPORTED.  BC vectors of
 * bcsrc changed since the last upload must fit the device table it already
 * has (else CN_ERR_INVALID_ARGUMENT: call cn_bc_sync first).  The first call
 * on a device looks the array up; calls that overlap on one device share the
 * array and race. */
cn_status cn_euler_rk3_stage_noalloc(cn_grid *bcsrc, cn_grid *Us, cn_grid *Un, cn_grid *out, int stage,
                                     double dt, double gamma, double *sums_out, void *stream);
/* U <- U^{n+1}: three stages through work1, work2 (same shape as U). */
cn_status cn_euler_rk3_step(cn_grid *U, cn_grid *work1, cn_grid *work2, double dt, double gamma,
                            double *sums_out, void *stream);
/* max over cells of |u_d| + c per direction (waits for the stream). */
cn_status cn_euler_max_speed(cn_grid *U, double gamma, double out[3], void *stream);

/* ------------------------------------------------------------ multigrid */
/* Geometric multigrid for div(k grad p) = f on a periodic grid (the
 * reference announces integrated multigrid solvers, README.rst:43-44, with
 * no code).  k: FLOAT32 cell coefficients, 1 component, cubic cells; the
 * levels halve the cells per block while they are even (max_levels <= 0: all).
 * Operator: harmonic face means, L p = ih2 * sum_d [kf+(p+ - p) - kf-(p - p-)];
 * smoother: weighted Jacobi (omega), nu1 pre / nu2 post sweeps; restriction:
 * mean of 8 children; prolongation: trilinear; coarsest level (<= 4096 cells):
 * FP64 conjugate gradients in one CTA.  V-cycles run in FP32. */
typedef struct cn_mg cn_mg;
cn_status cn_mg_create(cn_grid *k, int nu1, int nu2, double omega, int max_levels, cn_mg **out);
cn_status cn_mg_destroy(cn_mg *m);
cn_status cn_mg_levels(const cn_mg *m, int *nlevels, int *coarsest_cells);
/* e = one V-cycle for L e = rhs from e = 0 (FLOAT32 grids of the finest shape). */
cn_status cn_mg_vcycle(cn_mg *m, const cn_grid *rhs, cn_grid *e, void *stream);
/* FP64 residual r = f - L p64 (p64 FLOAT64, f FLOAT32); r32 optional FLOAT32
 * copy of r; returns sum r^2 and sum f^2 (waits for the stream). */
cn_status cn_mg_residual(cn_mg *m, const cn_grid *p64, const cn_grid *f, cn_grid *r32, double *rr,
                         double *ff, void *stream);
/* Solve to ||f - L p|| <= rtol ||f||: p64 zeroed, then per cycle the FP64
 * residual, one FP32 V-cycle on it, p64 += e (defect correction). */
cn_status cn_mg_solve(cn_mg *m, const cn_grid *f, cn_grid *p64, double rtol, int max_cycles,
                      int *cycles, double *relres, void *stream);
/* Single finest-level operators (tests): one Jacobi sweep, residual
 * restricted onto level 1, and p += prolongation of a level-1 correction. */
cn_status cn_mg_jacobi(cn_mg *m, const cn_grid *pin, const cn_grid *f, cn_grid *pout, void *stream);
cn_status cn_mg_restrict_residual(cn_mg *m, const cn_grid *p, const cn_grid *f, cn_grid *fc,
                                  void *stream);
cn_status cn_mg_prolong(cn_mg *m, const cn_grid *ec, cn_grid *p, void *stream);
/* Level grids owned by the solver: which = 0 solution, 1 right-hand side, 2 k. */
cn_status cn_mg_level_grid(cn_mg *m, int level, int which, cn_grid **out);

/* p64 += the finest-level correction of the last V-cycle. */
cn_status cn_mg_accumulate(cn_mg *m, cn_grid *p64, void *stream);

/* ------------------------------------------------------ learned smoother */
/* A learned 3x3x3 convolutional smoother (no reference counterpart; the
 * reference has no learned components): inputs x0 = -r/D (the Jacobi
 * correction, r = f - L p, D = -diag L), x1 = x0 ln k,
 * h1 = relu(conv(W1, x)) (2 -> 16 ch), h2 = relu(conv(W2, h1)) (16 -> 16),
 * y = conv(W3, h2) (16 -> 1); smoothing step p += omega*x0 + y.  Weights
 * [tap][cin][cout], tap = dx+1 + 3(dy+1) + 9(dz+1), FP32 master copy. */
typedef struct cn_nn cn_nn;
cn_status cn_nn_create(uint64_t seed, double omega, double init_scale, cn_nn **out);
cn_status cn_nn_destroy(cn_nn *nn);
int cn_nn_weight_count(void);
cn_status cn_nn_get_weights(const cn_nn *nn, float *host);
cn_status cn_nn_set_weights(cn_nn *nn, const float *host);
/* Training loss (1/B) sum_b ||r_b - A c_b||^2 / ||r_b||^2, c = omega x0 + y,
 * and its gradient, on device patches x [B][2][(P+8)^3], k [B][(P+2)^3],
 * r [B][P^3]; grad_out (optional, device or host) receives all weights'
 * gradients.  Waits for the stream if loss is requested. */
cn_status cn_nn_loss_grad(cn_nn *nn, const float *x, const float *k, const float *r, int B, int P,
                          double ih2, double *loss, float *grad_out, void *stream);
cn_status cn_nn_adam_step(cn_nn *nn, double lr, void *stream);
cn_status cn_nn_train(cn_nn *nn, const float *x, const float *k, const float *r, int npatches, int P,
                      double ih2, int epochs, int batch, double lr, uint64_t seed, double *last_loss,
                      void *stream);
/* Training patches from `cycles` plain V-cycles of m on L p = f: per cycle
 * `per_snapshot` random blocks of the finest residual before pre-smoothing
 * and after the coarse-grid correction (device outputs, see cn_nn_loss_grad). */
cn_status cn_mg_collect_patches(cn_mg *m, const cn_grid *f, int cycles, int per_snapshot, uint64_t seed,
                                float *x, float *k, float *r, int max_patches, int *count, void *stream);
/* Use the network instead of Jacobi on the levels set in level_mask (bit l);
 * nn == NULL restores Jacobi everywhere. */
cn_status cn_mg_set_smoother(cn_mg *m, cn_nn *nn, unsigned level_mask);
/* The same per smoothing phase: the network pre-smooths the levels in
 * pre_mask and post-smooths those in post_mask, with pre_apps / post_apps
 * applications (-1: nu1 / nu2 of cn_mg_create); Jacobi elsewhere.
 * cn_mg_set_smoother(m, nn, mask) is (mask, mask, -1, -1). */
cn_status cn_mg_set_smoother_phases(cn_mg *m, cn_nn *nn, unsigned pre_mask, unsigned post_mask, int pre_apps,
                                    int post_apps);
/* Grid inference precision: 1 (default) = BF16 activations and weights on
 * the tensor cores (tcgen05, FP32 accumulation) on levels whose block cells
 * are multiples of (16, 16, 4), else FP32; 0 = FP32 on the CUDA cores. */
cn_status cn_nn_set_inference(cn_nn *nn, int mode);
/* Training precision (cn_nn_loss_grad, cn_nn_train): 1 (default) = the
 * hidden 16 -> 16 layer's forward, data gradient and weight gradient on the
 * tensor cores (tcgen05, BF16 operands, FP32 accumulation) with BF16
 * activations and activation gradients, the first and last layers on the
 * CUDA cores in FP32 arithmetic; 0 = FP32 throughout on the CUDA cores.
 * A tensor-core kernel whose bounded wait ran out makes the call return
 * CN_ERR_DEVICE. */
cn_status cn_nn_set_training(cn_nn *nn, int mode);
/* One 3x3x3 convolution, 16 -> 16 channels, on the tensor cores: in and out
 * are device arrays [nblocks][cells][16] of BF16 (channels last, blocks and
 * cells in grid order), neighbours across blocks periodic; weights FP32
 * device [27][16][16] ([tap][cin][cout], rounded to BF16); optional ReLU.
 * Block cells must be multiples of (16, 16, 4). */
cn_status cn_conv3_bf16(const void *in, void *out, const int nblocks[3], const int block_cells[3],
                        const float *weights, int relu, void *stream);

/* ----------------------------------------------------- AMR block layouts */
/* Cubic blocks of uneven sizes on two refinement levels (ratio 2) tiling a
 * periodic unit box (the reference sketches level interfaces only in its notes,
 * test/sandbox/doc/notes/01_notes.md:192-196).  Block b: level[b] in {0, 1}
 * (cell size 2 or 1 level-1 units), cells[b] (a multiple of 8) per dimension,
 * origin[3b..3b+2] in level-1 units (multiples of 8); fine_extent = the box
 * in level-1 cells.  Data: ncomp components, blocks contiguous in block order.
 * Ghost cells: same level copy; coarse source: trilinear prolongation (3/4,
 * 1/4 weights, stencil clamped to the source block); fine source: mean of the
 * 8 children (conservative restriction). */
typedef struct cn_amr cn_amr;
cn_status cn_amr_create(int nblocks, const int *level, const int *cells, const int *origin, int fine_extent,
                        int ncomp, cn_dtype dtype, cn_amr **out);
/* The same on a periodic box of fine_extent[0] x [1] x [2] level-1 cells
 * (each a multiple of 8); cells stay cubic, h = cell size / fine_extent[0]
 * (the box is [0,1] x [0, Ly/Lx] x [0, Lz/Lx]).  cn_amr_create is the cubic
 * case. */
cn_status cn_amr_create_box(int nblocks, const int *level, const int *cells, const int *origin,
                            const int fine_extent[3], int ncomp, cn_dtype dtype, cn_amr **out);
cn_status cn_amr_destroy(cn_amr *a);
cn_status cn_amr_info(const cn_amr *a, int64_t *total_cells, int64_t *comp_stride, int *nitems);
cn_status cn_amr_block_offset(const cn_amr *a, int block, int64_t *offset);
cn_status cn_amr_data(cn_amr *a, int comp, void **device_ptr);
/* Dense lab (n+2*ghost)^3 of one block, face ghosts only (corners untouched). */
cn_status cn_amr_lab_fill(cn_amr *a, int comp, int ghost, int block, void *d_lab, void *stream);
/* Euler (5 components, periodic box) on the layout: stage 0 = RHS, 1..3 =
 * SSP-RK3 stages as cn_euler_rk3_stage; one persistent launch per stage over
 * the 8^3-tile work list of Us. */
cn_status cn_amr_rk3_stage(cn_amr *Us, cn_amr *Un, cn_amr *out, int stage, double dt, double gamma,
                           void *stream);
cn_status cn_amr_rk3_step(cn_amr *U, cn_amr *w1, cn_amr *w2, double dt, double gamma, void *stream);
/* Work-list order (0 block order, 1 largest blocks first, 2 Morton order of
 * tiles) and persistent grid (0: one CTA per work item). */
cn_status cn_amr_set_schedule(cn_amr *a, int order, int ctas);
/* Work tile of a CTA's work item: shape[d] in {1, 2, 4} 8^3 tiles along
 * x, y, z of one block (8x8x8 up to 32x32x32 cells, clipped to the block),
 * processed in turn by one CTA; the stage's compute tile stays 8^3.
 * cn_amr_set_work_unit(a, t) is the shape (t, 1, 1). */
cn_status cn_amr_set_work_shape(cn_amr *a, const int shape[3]);
cn_status cn_amr_set_work_unit(cn_amr *a, int tiles);
cn_status cn_amr_get_work_shape(const cn_amr *a, int shape[3]);
/* out = {order, ctas, tiles per work tile} of a layout. */
cn_status cn_amr_get_schedule(const cn_amr *a, int out[3]);
/* Times all schedules (orders x work-tile shapes x grid sizes) over `reps`
 * steps (advancing U) and keeps the fastest; the shape chosen is read back
 * with cn_amr_get_work_shape. */
cn_status cn_amr_autotune(cn_amr *U, cn_amr *w1, cn_amr *w2, double dt, double gamma, int reps,
                          int *order_out, int *ctas_out, double *ms_out, void *stream);

/* ----------------------------------------------------------- CUDA graphs */
/* Capture the calls issued on `stream` between begin and end into a graph
 * (thread-local capture).  Run each captured call once eagerly first, and
 * synchronise BC tables (cn_bc_sync) before capturing. */
typedef struct cn_graph cn_graph;
cn_status cn_graph_begin(void *stream);
cn_status cn_graph_end(void *stream, cn_graph **out);
cn_status cn_graph_launch(cn_graph *g, void *stream);
cn_status cn_graph_destroy(cn_graph *g);

/* ------------------------------------------------- pointwise field ops */
/* The optimised hooks that Block/FieldOperator.h:149-227 declares (under
 * CUBISM_OPTIMIZED_FIELD_OP) and never defines, with the reference's exact
 * names and signatures:  dst[i] = src0[i] OP src1[i]  (...2_T),
 * dst[i] = src0[i] OP src1  (...1_T),  fieldRcp: dst[i] = src1 * (1/src0[i])
 * (FieldOperator.h:16-30).  Device or managed pointers run in place, host
 * pointers are staged through device memory; each call returns once dst
 * holds the result. */
void fieldAdd2_double(const double *src0, const double *src1, double *dst, const size_t n);
void fieldSub2_double(const double *src0, const double *src1, double *dst, const size_t n);
void fieldMul2_double(const double *src0, const double *src1, double *dst, const size_t n);
void fieldDiv2_double(const double *src0, const double *src1, double *dst, const size_t n);
void fieldAdd2_float(const float *src0, const float *src1, float *dst, const size_t n);
void fieldSub2_float(const float *src0, const float *src1, float *dst, const size_t n);
void fieldMul2_float(const float *src0, const float *src1, float *dst, const size_t n);
void fieldDiv2_float(const float *src0, const float *src1, float *dst, const size_t n);
void fieldAdd1_double(const double *src0, const double src1, double *dst, const size_t n);
void fieldSub1_double(const double *src0, const double src1, double *dst, const size_t n);
void fieldMul1_double(const double *src0, const double src1, double *dst, const size_t n);
void fieldDiv1_double(const double *src0, const double src1, double *dst, const size_t n);
void fieldAdd1_float(const float *src0, const float src1, float *dst, const size_t n);
void fieldSub1_float(const float *src0, const float src1, float *dst, const size_t n);
void fieldMul1_float(const float *src0, const float src1, float *dst, const size_t n);
void fieldDiv1_float(const float *src0, const float src1, float *dst, const size_t n);
void fieldRcp_double(const double *src0, const double src1, double *dst, const size_t n);
void fieldRcp_float(const float *src0, const float src1, float *dst, const size_t n);
/* Stream-ordered form on device pointers: op 0..4 = add, sub, mul, div, rcp;
 * src1 == NULL selects the scalar form (rcp always uses the scalar). */
cn_status cn_field_op(int op, cn_dtype dtype, const void *src0, const void *src1, double scalar,
                      void *dst, size_t n, void *stream);

/* --------------------------------------------------------- calibration */
/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of the current device
 * for FLOAT64 or FLOAT32: the roofline denominator of the ALU-bound Euler
 * kernels.  No reference counterpart (the reference has no device code).
 * Synchronous; takes a few milliseconds. */
cn_status cn_calib_fma_peak(cn_dtype dtype, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* CUBISMNOVA_B200_H */
