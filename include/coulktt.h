/*
 * coulktt.h -- C ABI of the B200-native direct Coulomb summation library
 * (libcoulktt.so).
 *
 * This is the thin layer that KTT-style host code reaches through the C++
 * ktt::Tuner surface (include/Ktt.h), and that other languages bind directly
 * (Python ctypes in ktt_b200/__init__.py).  Plain pointers and sizes only; no
 * C++ or torch types cross it; no exception crosses it.  Every function
 * returns a coul_status; on failure a description is available from
 * coul_last_error() (thread-local).
 *
 * What each entry point replaces in KTT 2.1.0 (paths relative to the KTT tree):
 *   coul_ctx_create/destroy   Tuner::Tuner / ~Tuner on one CUDA device
 *                             (Source/Tuner.h:70, Source/ComputeEngine/Cuda/CudaEngine.cpp:29-60)
 *   coul_forward_3d           launch of directCoulombSum, 3D
 *                             (Examples/CoulombSum3d/CoulombSum3d.cu:1-47 through
 *                             Source/ComputeEngine/Cuda/CudaKernel.cpp:43-70)
 *   coul_forward_3d_soa       same with USE_SOA == 1 argument layout
 *                             (Examples/CoulombSum3d/CoulombSum3d.cu:23-28)
 *   coul_forward_3d_reference launch of directCoulombSumReference
 *                             (Examples/CoulombSum3d/CoulombSum3dReference.cu:1-28)
 *   coul_forward_2d           launch of directCoulombSum, 2D slice with the
 *                             precomputed dz^2 in the atom's .z
 *                             (Examples/CoulombSum2d/CoulombSum2dSimple.cl:29-79,
 *                             reference Examples/CoulombSum2d/CoulombSum2dReference.cl:1-21)
 *   coul_slice_atoms          the host-side dz^2 precompute of the iterative
 *                             launcher (Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp:160-179),
 *                             done on the device
 *   coul_forward_3d_host      Tuner::Run with host output buffers
 *                             (Source/Tuner.h:536, BufferOutputDescriptor download)
 *   coul_elapsed_ms           kernel duration from the event pair bracketing the launch
 *                             (Source/ComputeEngine/Cuda/CudaKernel.cpp:62-67, CudaEvent.cpp:30-36)
 *   coul_synchronize          ComputeInterface::SynchronizeQueue / WaitForComputeAction
 *                             (Source/Api/ComputeInterface.h)
 *   coul_tune_supported       the CompilationFailed / DeviceLimitsExceeded checks made before a
 *                             launch (Source/ComputeEngine/Cuda/CudaEngine.cpp:117-138); here a
 *                             configuration maps onto an ahead-of-time compiled sm_100a variant
 *
 * Units and layout: atoms are float4 (x, y, z, q) in Angstrom / elementary
 * charge, 16-byte aligned; grid point (i, j, k) sits at
 * (fmaf(i, h, ox), fmaf(j, h, oy), fmaf(k, h, oz)) -- for a zero origin this
 * is KTT's gridSpacing * index; the map is stored x fastest:
 * out[(k * ny + j) * nx + i].  Pointers named d_* are device pointers, h_*
 * host pointers.  All launches are asynchronous on the context's stream
 * unless stated otherwise.
 */
#ifndef COULKTT_H
#define COULKTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define COUL_API __attribute__((visibility("default")))
#else
#define COUL_API
#endif

typedef enum coul_status {
    COUL_OK = 0,
    COUL_ERR_INVALID_ARGUMENT = 1,  /* bad pointer, size, alignment or grid */
    COUL_ERR_CUDA = 2,              /* a CUDA runtime call failed */
    COUL_ERR_UNSUPPORTED = 3,       /* no compiled variant for this configuration (KTT: CompilationFailed) */
    COUL_ERR_DEVICE_LIMITS = 4,     /* block size / shared memory beyond the device (KTT: DeviceLimitsExceeded) */
    COUL_ERR_TIMEOUT = 5,           /* a bounded device-side wait gave up; results are invalid */
    COUL_ERR_NO_DEVICE = 6,         /* no CUDA device, or not an sm_100 device */
    COUL_ERR_OUT_OF_MEMORY = 7
} coul_status;

/* Where the atom stream is read from inside the kernel (KTT USE_CONSTANT_MEMORY). */
enum {
    COUL_ATOMS_SHARED_TMA = 0, /* tiles staged into shared memory by TMA bulk copies */
    COUL_ATOMS_CONSTANT = 1    /* chunks of 4096 atoms copied into __constant__ memory */
};

/* Precision form.  FP32, compensated and both FP64 merges evaluate each pair in FP32 and differ in
   how they accumulate; FP64 pairs evaluates each pair in FP64. */
enum {
    COUL_PREC_FP32 = 0,        /* one FP32 accumulator per point (KTT's kernel) */
    COUL_PREC_COMPENSATED = 1, /* FP32 partial per 64-atom sub-tile, merged by two-sum into (sum, error) */
    COUL_PREC_FP64_MERGE = 2,  /* FP32 partial per 64-atom sub-tile, merged into an FP64 accumulator */
    COUL_PREC_FP64_PAIRS = 3,  /* every pair in FP64: exact differences, FP64 r^2, MUFU rsqrt estimate
                                  refined by one FP64 Newton step (about 2^-40), FP64 accumulation; the
                                  map's error is then its FP32 store.  3D maps, rsqrt_soft 0 only */
    COUL_PREC_FP64_MERGE_SHARED = 4 /* COUL_PREC_FP64_MERGE with the FP64 sums in shared memory instead of
                                       registers (8 bytes per point per thread): the same values bit for
                                       bit, more resident warps.  3D maps, TMA-staged atoms */
};

/*
 * Tuning parameters of the forward kernel.  The names in brackets are the KTT
 * tuning parameters of Examples/CoulombSum3d/CoulombSum3d.cpp:137-216 that
 * map onto each field.
 */
typedef struct coul_tune {
    int block_x;      /* threads per block along x             [WORK_GROUP_SIZE_X] */
    int block_y;      /* threads per block along y             [WORK_GROUP_SIZE_Y] */
    int z_iterations; /* grid points per thread along z         [Z_ITERATIONS] (3D); along y for 2D */
    int x_points;     /* grid points per thread along x, stored as one float/float2/float4 vector
                                                               [VECTOR_SIZE; OUTER_UNROLL_FACTOR in 2D] */
    int unroll;       /* unroll of the atom loop; 0 and 1 mean none [INNER_UNROLL_FACTOR] */
    int atom_source;  /* COUL_ATOMS_*                          [USE_CONSTANT_MEMORY] */
    int precision;    /* COUL_PREC_* */
    int rsqrt_soft;   /* share of the reciprocal square roots taken on the FMA pipe (Newton
                         iterations) instead of the MUFU unit, in eighths (0 = all MUFU).  A thread
                         evaluates x_points * z_iterations points per atom in n lane pairs; within one
                         stage of 256 atoms each pair keeps one form for every atom.  With n >= 8, pair
                         p is on the FMA pipe when (p % 8) < rsqrt_soft; with n < 8 the stages (in
                         the atom-split form also the warps of a block) take turns in 8 / n phases
                         and pair p in phase g is on the FMA pipe when g * n + p < rsqrt_soft.  Either
                         way the share is rsqrt_soft / 8.
                         10 + k (k = 0..7): successive patterns alternate between k and k + 1 eighths,
                         a share of (2k + 1) / 16 */
    int atom_split;   /* 0 or 1: one CTA per point tile; 2 or more: the atoms are split into that
                         many chunks per point tile, the partial sums of a tile added in chunk order
                         (for slices and small maps with too few tiles to fill the GPU; FP32,
                         shared-memory atoms).  How, is split_form's choice */
    int split_form;   /* with atom_split >= 2: 0 = a thread-block cluster of atom_split CTAs (2..16;
                         above 8 a non-portable size, refused with COUL_ERR_DEVICE_LIMITS where the
                         block does not fit) reduces its partial blocks over distributed shared
                         memory; 1 = a persistent grid (as many CTAs as fit) claims (tile, chunk)
                         items from a device queue and the CTA finishing a tile's last chunk adds the
                         tile's partial blocks from device memory (atom_split 2..256; no clusters, so
                         every SM gets the same share of the work; the context keeps the partial
                         blocks, 4 bytes per point per chunk); 2 = balanced: a resident grid whose
                         CTAs take equal contiguous ranges of the (point tile, atom) space, each CTA
                         block_x x block_y x atom_split threads (at most 1024; atom_split 2..32 groups
                         that share the tile's points and split every atom stage), a tile split
                         between CTAs finished from device memory by the CTA adding its last piece */
} coul_tune;

typedef struct coul_grid {
    int nx, ny, nz;    /* points along each axis (nz = 1 for a single slice) */
    float spacing;     /* h, Angstrom */
    float origin[3];   /* coordinate of point (0, 0, 0) */
} coul_grid;

typedef struct coul_ctx coul_ctx;

/* ---- context ------------------------------------------------------------ */
COUL_API int coul_ctx_create(int device, coul_ctx** ctx);
/* Also releases the device resources of the context's batches that are still alive; their handles
   stay valid for coul_batch_destroy only (coul_batch_run refuses them). */
COUL_API int coul_ctx_destroy(coul_ctx* ctx);
/* A context on the caller's own CUDA context (a CUcontext, passed as void*) instead of the device's
   primary context: every later call of this context makes cu_context current on the calling thread.
   `stream` (a CUstream of that context, or NULL for a stream of its own) is where calls are
   enqueued.  The caller keeps ownership of both and destroys them after coul_ctx_destroy.  Replaces
   KTT's CUDA engine set-up from a ComputeApiInitializer (Source/ComputeEngine/Cuda/CudaEngine.cpp:67-106,
   Source/Api/ComputeApiInitializer.h:26). */
COUL_API int coul_ctx_create_on(void* cu_context, void* stream, coul_ctx** ctx);
/* Enqueue every later call of this context on the given cudaStream_t (passed as void*).  NULL is
   the legacy default stream (PyTorch's default stream), not a private one.  A new context starts
   on a non-blocking stream of its own, returned by coul_ctx_own_stream. */
COUL_API int coul_ctx_set_stream(coul_ctx* ctx, void* stream);
COUL_API void* coul_ctx_get_stream(coul_ctx* ctx);
COUL_API void* coul_ctx_own_stream(coul_ctx* ctx);
/* Index of the context's CUDA device. */
COUL_API int coul_ctx_device(coul_ctx* ctx, int* device);
/* Number of SMs and compute capability of the context's device. */
COUL_API int coul_ctx_device_info(coul_ctx* ctx, int* sm_count, int* cc_major, int* cc_minor);

/* Properties of a CUDA device, without a context: what KTT's CUDA engine reads with
   cuDeviceGetName / cuDeviceTotalMem / cuDeviceGetAttribute for its DeviceInfo
   (Source/ComputeEngine/Cuda/CudaDevice.cpp:26-58) and cuDriverGetVersion for its PlatformInfo
   (CudaEngine.cpp:696-707). */
typedef struct coul_device_props {
    char name[256];
    uint64_t global_memory;        /* bytes */
    uint64_t shared_memory_block;  /* bytes of shared memory per block without opt-in (KTT: local memory) */
    uint64_t constant_memory;      /* bytes */
    int max_threads_block;         /* KTT: maximum work-group size */
    int sm_count;
    int cc_major, cc_minor;
    int driver_version;            /* cudaDriverGetVersion, e.g. 12090 */
} coul_device_props;
/* Number of CUDA devices (0 with no device or no driver: returns COUL_OK). */
COUL_API int coul_device_count(int* count);
COUL_API int coul_device_query(int device, coul_device_props* props);
/* Wait for the context's stream; returns COUL_ERR_TIMEOUT if a kernel reported a bounded-wait expiry. */
COUL_API int coul_synchronize(coul_ctx* ctx);
/* Duration in ms between the events bracketing the most recent forward/adjoint/batched call
   (waits for it).  With several launches in one call the span covers all of them. */
COUL_API int coul_elapsed_ms(coul_ctx* ctx, double* ms);
/* Thread-local message for the last failing call on this thread ("" if none). */
COUL_API const char* coul_last_error(void);
COUL_API const char* coul_status_string(int status);

/* ---- device buffers --------------------------------------------------------- */
/*
 * Device memory for hosts that do not hold a CUDA runtime of their own (the C++ ktt::Tuner
 * surface keeps kernel arguments through these; KTT's CUDA engine does the same with its
 * CudaBuffer class, Source/ComputeEngine/Cuda/Buffers/CudaBuffer.cpp).  Copies are ordered on the
 * context's stream; upload/download of pageable host memory return when the copy is done.
 */
COUL_API int coul_buffer_alloc(coul_ctx* ctx, size_t bytes, void** d_ptr);
COUL_API int coul_buffer_free(coul_ctx* ctx, void* d_ptr);
COUL_API int coul_buffer_upload(coul_ctx* ctx, void* d_dst, const void* h_src, size_t bytes);
COUL_API int coul_buffer_download(coul_ctx* ctx, void* h_dst, const void* d_src, size_t bytes);
COUL_API int coul_buffer_copy(coul_ctx* ctx, void* d_dst, const void* d_src, size_t bytes);
COUL_API int coul_buffer_memset(coul_ctx* ctx, void* d_dst, int value, size_t bytes);

/* ---- tuning parameters ---------------------------------------------------- */
COUL_API void coul_tune_default(coul_tune* tune);
/* COUL_OK if the configuration maps to a compiled kernel variant that fits the device. */
COUL_API int coul_tune_supported(const coul_tune* tune);
/* The same check for coul_forward_2d (2D-slice variants). */
COUL_API int coul_tune_supported_2d(const coul_tune* tune);
/* Number of compiled forward variants, and the i-th one (for the tuner's space checks): its
   tuning fields (block shape left at the default), whether it is a 2D-slice variant, and whether
   it reads the four-array atom layout. */
COUL_API int coul_variant_count(void);
COUL_API int coul_variant_get(int i, coul_tune* tune, int* is_2d, int* is_soa);

/* ---- forward: potential map -------------------------------------------------- */
/*
 * 3D map on a regular grid.  accumulate = 0 writes out = V; accumulate = 1
 * adds (out += V, KTT's kernel semantics: the grid is zeroed by the caller).
 */
COUL_API int coul_forward_3d(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                             const coul_tune* tune, int accumulate, float* d_out);
/*
 * One z slab of the 3D map: the points z in [z_begin, z_end) of the full grid `grid`, written to
 * d_out as (z_end - z_begin) x ny x nx values (x fastest).  The points' coordinates are those of
 * the full grid, so the slabs of a z-sharded map (one per GPU) put together equal the single-GPU
 * map bit for bit when every z_begin is a multiple of tune->z_iterations (otherwise a point may
 * take its rsqrt from the other pipe and differ in the last bits).  No counterpart in the reference (KTT runs one map per kernel launch); it is
 * the sharding unit of the multi-GPU path.
 */
COUL_API int coul_forward_3d_slab(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                                  int z_begin, int z_end, const coul_tune* tune, int accumulate, float* d_out);
/* Same with the atom coordinates and charges in four separate arrays. */
COUL_API int coul_forward_3d_soa(coul_ctx* ctx, const float* d_x, const float* d_y, const float* d_z,
                                 const float* d_q, int64_t n_atoms, const coul_grid* grid, const coul_tune* tune,
                                 int accumulate, float* d_out);
/*
 * One grid point per thread, atoms read straight from global memory, FP32
 * accumulation: the semantics of KTT's reference kernel (out += V).  Kept as
 * a cross-check and as the "plain launch" baseline of the tuner.
 */
COUL_API int coul_forward_3d_reference(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms,
                                       const coul_grid* grid, int accumulate, float* d_out);
/*
 * The same map evaluated in FP64 on the GPU, for validating configurations while tuning (KTT's
 * Coulomb examples validate against a reference kernel, Examples/CoulombSum3d/CoulombSum3d.cpp:
 * 221-227; KTT registers CPU reference computations through Tuner::SetReferenceComputation,
 * Source/Tuner.h:610).  One point per thread; the FP32 grid coordinates (as the tiled kernels form
 * them) and atoms widened to double, then differences, squares, square root and division in FP64,
 * accumulated in FP64; d_out holds nx * ny * nz doubles (assigned).  Slow (no MUFU, no register
 * blocking): a checker, not a product form.
 */
COUL_API int coul_forward_3d_reference_fp64(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms,
                                            const coul_grid* grid, double* d_out);
/*
 * 2D slice in KTT's 2D argument convention: d_atoms holds (x, y, dz2, q) with
 * dz2 the squared z distance of the atom to the slice.  out[j*nx + i] over an
 * nx * ny slice with spacing h and zero origin.  tune->z_iterations is the
 * register block along y, tune->x_points along x.
 */
COUL_API int coul_forward_2d(coul_ctx* ctx, const float* d_atoms_xy_dz2_q, int64_t n_atoms, float spacing, int nx,
                             int ny, const coul_tune* tune, int accumulate, float* d_out);
/* Gather four separate atom arrays (KTT's USE_SOA layout: atomInfoX/Y/Z/W) into float4 (x, y, z, q),
   on the device; d_out must hold n_atoms float4 and be 16-byte aligned.  d_q may be NULL: the
   fourth component is then 0 (three-component arrays such as N-body velocities). */
COUL_API int coul_pack_atoms(coul_ctx* ctx, const float* d_x, const float* d_y, const float* d_z, const float* d_q,
                             int64_t n_atoms, float* d_out);
/* Convert (x, y, z, q) atoms into the 2D convention (x, y, (z_slice - z)^2, q) on the device. */
COUL_API int coul_slice_atoms(coul_ctx* ctx, const float* d_xyzq, int64_t n_atoms, float z_slice,
                              float* d_xy_dz2_q);
/*
 * Host-buffer convenience call: uploads h_atoms, computes the 3D map (out = V)
 * and downloads it into h_out, then waits.  Device buffers are cached in the
 * context and grown on demand.
 */
COUL_API int coul_forward_3d_host(coul_ctx* ctx, const float* h_atoms, int64_t n_atoms, const coul_grid* grid,
                                  const coul_tune* tune, float* h_out);

/* ---- adjoint: gradient of a loss on the map ----------------------------------------- */
/*
 * Given G = dL/dV on the nx*ny*nz grid (d_grad_map, x fastest) for the map of coul_forward_3d,
 * writes d_grad_q[j] = dL/dq_j = sum_i G_i / r_ij and d_grad_xyz[3j..3j+2] = dL/dr_j =
 * q_j sum_i G_i (r_i - r_j) / r_ij^3 (either output may be NULL).  1/r is recomputed, nothing is
 * stored per pair; partial sums are FP64 and added in a fixed order (deterministic).  For the weighted
 * least-squares loss L = 0.5 sum_i w_i (V_i - T_i)^2 pass G_i = w_i (V_i - T_i).  No counterpart in KTT
 * (it tunes forward kernels only); the PyTorch binding wraps forward + adjoint as an autograd function.
 * Asynchronous on the context's stream; keeps an FP64 workspace of 32 * n_atoms * chunks bytes in the
 * context (chunks ~ 24 * SMs / atom tiles).
 */
COUL_API int coul_adjoint_3d(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                             const float* d_grad_map, float* d_grad_q, float* d_grad_xyz);

/* ---- N-body: the sibling pair sum of KTT's Nbody example ---------------------------------- */
/* Tuning fields (the KTT parameter each one covers in brackets, Examples/Nbody/Nbody.cpp:140-209). */
typedef struct coul_nbody_tune {
    int block_x;           /* threads per block, a multiple of 32 up to 512      [WORK_GROUP_SIZE_X] */
    int bodies_per_thread; /* bodies i per thread in registers: 1, 2, 4 or 8     [OUTER_UNROLL_FACTOR] */
    int unroll;            /* unroll of the loop over bodies j: 1, 2 or 4        [INNER_UNROLL_FACTOR1] */
    int j_split;           /* 0 / 1: one CTA per tile of bodies i; 2..16: a thread-block cluster of that
                              many CTAs shares the tile, each taking a share of the bodies j, partial
                              accelerations reduced over distributed shared memory; above 8 a
                              non-portable cluster size, refused with COUL_ERR_DEVICE_LIMITS where the
                              blocks do not fit such a cluster                  [WORK_GROUP_SIZE_Y] */
} coul_nbody_tune;
COUL_API int coul_nbody_tune_default(coul_nbody_tune* tune);
COUL_API int coul_nbody_tune_supported(const coul_nbody_tune* tune);
/*
 * One step of KTT's nbody_kernel (Examples/Nbody/Nbody.cu:260-410; reference NbodyReference.cu:36-75):
 * for every body i, a_i = sum_j m_j d_ij / (|d_ij|^2 + softening_sqr)^(3/2) with d_ij = p_j - p_i,
 * then p_i' = p_i + dt v_i + damping dt^2 a_i and v_i' = v_i + dt a_i.  d_pos_mass holds n float4
 * (x, y, z, mass), d_vel n float4 (x, y, z, unused); the outputs (16-byte aligned, not aliasing the
 * inputs) get (x', y', z', mass) and (vx', vy', vz', 0).  Any n >= 0 (KTT's kernel needs n to be a
 * multiple of its tile).  Asynchronous on the context's stream; timed by coul_elapsed_ms.
 */
COUL_API int coul_nbody_step(coul_ctx* ctx, const float* d_pos_mass, const float* d_vel, int64_t n, float dt,
                             float damping, float softening_sqr, const coul_nbody_tune* tune, float* d_pos_mass_new,
                             float* d_vel_new);

/* ---- batched: many molecules in one persistent launch ------------------------------ */
/*
 * A batch of molecules with uneven atom counts and grids, computed by one persistent launch that
 * pulls (molecule, tile) work items from a device queue, molecules in decreasing order of pair
 * count.  Replaces the one-launch-per-problem pattern of KTT's custom launchers
 * (Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp:146-184).  The batch keeps the
 * molecule table and the queue counter on the device; the caller keeps its atom and output
 * buffers alive while the batch exists.
 */
typedef struct coul_molecule {
    const float* d_atoms; /* n_atoms float4 (x, y, z, q), 16-byte aligned */
    int64_t n_atoms;
    coul_grid grid;
    float* d_out;         /* nx * ny * nz floats, x fastest */
} coul_molecule;

typedef struct coul_batch coul_batch;

enum {
    COUL_BATCH_PERSISTENT = 0, /* queue reset + one persistent launch */
    COUL_BATCH_GRAPH = 1,      /* the same two steps captured once into a CUDA graph and replayed */
    COUL_BATCH_SEPARATE = 2    /* baseline: one plain forward launch per molecule */
};

/* Whether a persistent batched variant is compiled for this tile shape (the batch's counterpart of
   coul_tune_supported). */
COUL_API int coul_batch_tune_supported(const coul_tune* tune);
/* tune selects the tile shape (z_iterations, x_points, unroll, precision, rsqrt_soft, block).  With
   x_points 1 the tiles are linear in each molecule's x-y plane (thread i of x-y tile j takes the
   plane's point j * threads + i, row-major), so only the plane's last tile is padded; otherwise the
   block's threads are arranged per molecule as the power-of-two x extent that pads the plane least.
   COUL_BATCH_SEPARATE launches the forward kernel of the same tune, which needs its own variant. */
COUL_API int coul_batch_create(coul_ctx* ctx, const coul_molecule* molecules, int n_molecules, const coul_tune* tune,
                               coul_batch** batch);
COUL_API int coul_batch_destroy(coul_batch* batch);
/* Enqueue one evaluation of every molecule's map (accumulate as in coul_forward_3d); timed like
   the forward calls (coul_elapsed_ms covers the whole batch). */
COUL_API int coul_batch_run(coul_ctx* ctx, coul_batch* batch, int mode, int accumulate);
COUL_API int coul_batch_info(const coul_batch* batch, int64_t* work_items, int* grid_ctas, double* total_pairs);

/*
 * The batched map without any device allocation.  No counterpart in the reference (KTT allocates
 * a buffer for every kernel argument).  For callers that must not allocate device memory from a
 * library: a host application that gives all free device memory to its own pool at start-up, a
 * latency-critical loop that cannot take the device-wide synchronisation of cudaFree, a plug-in
 * whose host owns every allocation.  Computes the same maps as coul_batch_create + coul_batch_run
 * (COUL_BATCH_PERSISTENT) on the current device and the given cudaStream_t (NULL = legacy default
 * stream), but keeps the work-queue counter and the molecule table in a fixed static device array
 * of the library (73,984 bytes, held by every GPU that loads the library until the process exits) and
 * calls no cudaMalloc, cudaFree or other allocating routine.  The caller passes the atom and output
 * buffers as in coul_molecule, and optionally d_status, an int in device memory that the kernel sets
 * to non-zero if a bounded device-side wait expires (the caller clears it).
 *   - at most 1024 molecules per call (larger batches are rejected with COUL_ERR_INVALID_ARGUMENT);
 *   - tile shapes (z_iterations/x_points/unroll/precision/rsqrt_soft, any block up to 256 threads):
 *     8/2/2/0/2, 8/2/1/0/0, 16/1/1/0/2; others return COUL_ERR_UNSUPPORTED;
 *   - the array exists once per CUDA context that loads the library (the device's primary context,
 *     or a context of the caller's own, current on the calling thread); every call looks up its
 *     device address in the current context (cudaGetSymbolAddress, a lookup that allocates
 *     nothing).  The first call in a context also loads the library's device code into it: make
 *     that first call before any stream capture;
 *   - every call shares the one array and leaves its table behind; calls whose kernels overlap on
 *     the GPU (different streams without ordering) race on it and give wrong maps.
 * Returns after enqueueing (the molecule table is copied from host memory before it returns).
 */
COUL_API int coul_batch_run_static(void* stream, const coul_molecule* molecules, int n_molecules,
                                   const coul_tune* tune, int accumulate, int* d_status);

/* ---- roofline ------------------------------------------------------------------ */
/*
 * Measures, on the context's device at its current clocks, the whole-GPU rate of MUFU reciprocal
 * square roots and of FP32 FMAs (operations per second) with two throughput microkernels.  The
 * pair-evaluation rooflines follow from them: all-MUFU R_mufu = rsqrt_per_s; with a share of the
 * rsqrts moved to the FMA pipe at s issue slots each, R_comb = rsqrt_per_s * (F/M - 1 + s) / (2 + s)
 * with F/M = ffma_per_s / rsqrt_per_s.  (KTT reads pipe utilisation from CUPTI instead:
 * Source/ComputeEngine/Cuda/Cupti/CuptiMetricInterface.cpp:621-660.)
 */
COUL_API int coul_measure_pipe_rates(coul_ctx* ctx, double* rsqrt_per_s, double* ffma_per_s);

/* The same microkernels and three more, reported separately (no counterpart in the reference):
 *   rsqrt_per_s        MUFU rsqrt.approx.f32 results per second;
 *   ffma_per_s         FP32 FMAs per second issued as scalar FFMA;
 *   ffma2_lanes_per_s  FP32 FMAs per second issued as packed FFMA2 (two per instruction), the form
 *                      the pair kernels use; coul_measure_pipe_rates reports the larger of the two;
 *   dfma_per_s         FP64 FMAs per second;
 *   rsqrt_mix6_per_s   MUFU rsqrts per second when six independent FP32 FMAs issue beside each one
 *                      (with one issue slot per MUFU instruction this would equal rsqrt_per_s; the
 *                      drop measures what a MUFU instruction costs in issue slots);
 *   sm_count, max_sm_clock_khz  the device's SM count and its maximum SM clock, for the datasheet
 *                      lane rates (128 FP32 lanes and 16 MUFU results per SM per clock on sm_100). */
typedef struct coul_pipe_rates {
    double rsqrt_per_s;
    double ffma_per_s;
    double ffma2_lanes_per_s;
    double dfma_per_s;
    double rsqrt_mix6_per_s;
    int sm_count;
    int max_sm_clock_khz;
} coul_pipe_rates;
COUL_API int coul_measure_pipe_rates_ex(coul_ctx* ctx, coul_pipe_rates* out);

/* ---- hardware counters ----------------------------------------------------------- */
/*
 * Counter collection around the context's launches with CUPTI's range profiler (user range,
 * user replay), loaded at run time from libcupti.  Replaces KTT's CUPTI metric interface
 * (Source/ComputeEngine/Cuda/Cupti/CuptiMetricInterface.cpp:21-120: metric configuration,
 * counter-data image, unsupported metrics dropped with a warning; CuptiInstance.cpp / CuptiPass:
 * one pass per kernel run, repeated until every pass is collected).  Usage:
 *
 *   coul_profiler_create(ctx, names, n, valid, &p, &passes)   names the metrics (Perfworks names)
 *   do {                                               the caller reruns the same launches once per
 *       coul_profiler_begin_pass(p);                   pass; they must do the same work each time
 *       ... launches on the context's stream ...
 *       coul_profiler_end_pass(p, &done);
 *   } while (!done);
 *   coul_profiler_read(p, values);                     one double per metric, in the given order
 *   coul_profiler_destroy(p);
 *
 * Metrics the device does not offer are dropped (valid[i] = 0, optional array of n entries) and
 * read back as NaN; if none is left, create fails with COUL_ERR_INVALID_ARGUMENT.  Clocks and other
 * device settings are left as they are.  One profiler per process at a time.  Without libcupti
 * create returns COUL_ERR_UNSUPPORTED.  coul_profiler_supported answers the same question without
 * a GPU for a named chip ("GB100" for B200).
 */
typedef struct coul_profiler coul_profiler;
COUL_API int coul_profiler_supported(const char* chip, const char* const* metrics, int n_metrics, int* valid);
COUL_API int coul_profiler_create(coul_ctx* ctx, const char* const* metrics, int n_metrics, int* valid,
                                  coul_profiler** out, int* passes);
COUL_API int coul_profiler_begin_pass(coul_profiler* profiler);
COUL_API int coul_profiler_end_pass(coul_profiler* profiler, int* all_passes_done);
COUL_API int coul_profiler_read(coul_profiler* profiler, double* values);
COUL_API int coul_profiler_destroy(coul_profiler* profiler);

/* ---- failure detection ------------------------------------------------------ */
/*
 * Runs one CTA that waits on an mbarrier with the given budget (at most 2 s).  With arrive != 0
 * the barrier completes and the call returns COUL_OK; with arrive == 0 nothing arrives, the
 * bounded wait expires, the kernel records the expiry in the context's status word and exits, and
 * the call returns COUL_ERR_TIMEOUT with the context still usable.  This exercises the same
 * bounded-wait and status path every kernel of the library uses (KTT has no counterpart: its
 * failures surface as ResultStatus::ComputationFailed, Source/Api/Output/ResultStatus.h:12-33).
 */
COUL_API int coul_probe_bounded_wait(coul_ctx* ctx, int arrive, uint64_t budget_ns);

#ifdef __cplusplus
}
#endif

#endif /* COULKTT_H */
