/*
 * bem_b200.h -- C ABI of the B200 boundary-element library (libbemb200.so).
 *
 * Dense complex Helmholtz Galerkin BEM on triangle meshes in the P1 vertex
 * basis: single-/double-layer (and adjoint-double, hypersingular,
 * Burton-Miller) matrix assembly, the exterior-Neumann solve and
 * boundary-to-listener evaluation.  It replaces the pybind module that the
 * NeuralAT reference JIT-builds from src/bem/cuda/bind.cu (bindings at
 * bind.cu:178-223, loader src/bem/solver.py:9-31).
 *
 * Conventions
 *  - All array arguments are DEVICE pointers on the current CUDA device,
 *    unless a comment says "host".
 *  - vertices: float32 (nv, 3) row-major; triangles: int32 (nt, 3) row-major.
 *  - Complex arrays are interleaved complex64 (re, im) unless marked complex128.
 *  - Matrices are row-major: entry (a, b) at a * nv + b, rows = test-triangle
 *    vertices, columns = trial-triangle vertices (bind.cu:144-151).
 *  - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 *    stream).  Functions return a bem_status; 0 = success.  Functions that
 *    must inspect data on the host (geometry set-up, solver convergence)
 *    synchronise `stream`; all others are asynchronous.
 *  - The library never allocates device memory for outputs: the caller
 *    passes every output and workspace buffer.  Workspace sizes are queried
 *    with the *_bytes functions.
 *  - The library has no CPU fallback: without a usable CUDA device every
 *    entry point returns BEM_ERR_CUDA.
 */
#ifndef BEM_B200_H
#define BEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* bem_stream_t; /* cudaStream_t */

typedef enum bem_status {
  BEM_OK = 0,
  BEM_ERR_INVALID_ARGUMENT = 1, /* null pointer, negative size, unknown enum */
  BEM_ERR_INDEX = 2,            /* triangle vertex index outside [0, nv) */
  BEM_ERR_DEGENERATE = 3,       /* zero-area triangle or repeated vertex */
  BEM_ERR_WORKSPACE = 4,        /* workspace missing, too small or not built */
  BEM_ERR_NONFINITE = 5,        /* NaN / Inf in an input */
  BEM_ERR_NOT_CONVERGED = 6,    /* iteration limit reached before tolerance */
  BEM_ERR_BREAKDOWN = 7,        /* Krylov breakdown / singular system */
  BEM_ERR_CUDA = 8,             /* CUDA runtime error (incl. no device) */
  BEM_ERR_UNSUPPORTED = 9       /* valid request the library does not support */
} bem_status;

/* Operator types, same order as the reference's PotentialType
 * (src/bem/cuda/include/potential.h:7-15). */
enum {
  BEM_SINGLE_LAYER = 0,
  BEM_DOUBLE_LAYER = 1,
  BEM_ADJOINT_DOUBLE_LAYER = 2,
  BEM_HYPERSINGULAR = 3,
  BEM_BM_LHS = 4,
  BEM_BM_RHS = 5
};

/* Quadrature orders: (singular Gauss-Legendre points per dimension,
 * regular triangle-rule points), bind.cu:180-215. */
enum {
  BEM_ORDER_EXACT = 0,    /* <4,6>  "*_boundary_matrix"          */
  BEM_ORDER_APPROX = 1,   /* <2,3>  "*_boundary_matrix_approx"   */
  BEM_ORDER_APPROX_1 = 2  /* <2,1>  "*_boundary_matrix_approx_1" */
};

/* Human-readable name of a status code (static string). */
const char* bem_status_string(int status);
/* Library version string (static). */
const char* bem_version(void);
/* Number of kernels this library has launched in this process (host-side
 * counter, incremented at every launch site). */
unsigned long long bem_kernel_launches(void);

/* ------------------------------------------------------------------------
 * Geometry.  Replaces the per-call mesh handling of bind.cu:49-66 and the
 * Python preprocess (src/bem/solver.py:40-58): validates the mesh, computes
 * unit normals, surface curls, quadrature points, a locality-sorted triangle
 * order with 16-triangle tiles, and the touching-pair lists (the reference
 * rediscovers these by an O(T^2) scan in every call, bind.cu:81-97).
 * Both calls copy the mesh to the host and synchronise `stream`.
 * ---------------------------------------------------------------------- */
int bem_geometry_bytes(const float* vertices, int nv, const int* triangles, int nt, size_t* bytes,
                       bem_stream_t stream);
int bem_geometry_build(const float* vertices, int nv, const int* triangles, int nt, void* geom,
                       size_t geom_bytes, bem_stream_t stream);
/* Copies the per-triangle unit normals (nt,3) and surface curls (nt,3,3)
 * (rows b: n x grad phi_b), solver.py:40-58.  Either output may be NULL. */
int bem_geometry_normals(const void* geom, float* normals, float* curls, bem_stream_t stream);
/* BEM_OK, or BEM_ERR_CUDA if a bounded wait of an assembly kernel (the bulk
 * copies of trial tiles) expired while assembling on this geometry since the
 * last call; a matrix assembled meanwhile may be wrong.  The status word lives
 * in the geometry workspace (assembly kernels write it although the geometry
 * is passed as const); this call clears it and synchronises `stream`.  No
 * counterpart in the reference, whose kernels report no errors. */
int bem_geometry_status(const void* geom, bem_stream_t stream);
/* Forgets the host-side copy of the geometry header that the library keeps
 * per workspace address.  Call it before freeing or reusing a geometry
 * workspace; a later call that passes the same address then reads the header
 * from the device again (and rejects a buffer that holds no geometry with
 * BEM_ERR_WORKSPACE).  No counterpart in the reference. */
int bem_geometry_release(const void* geom);

/* ------------------------------------------------------------------------
 * Assembly on a built geometry.
 * ---------------------------------------------------------------------- */

/* Dense nv x nv Galerkin matrix of `layer` at quadrature `order`,
 * overwriting `out` (complex64).  Replaces the 18 assemble_matrix
 * bindings, bind.cu:49-154,180-215.  `normals`/`curls` (may be NULL: the
 * geometry's own) are the per-triangle arrays the reference passes in for
 * the hypersingular and Burton-Miller operators (bind.cu:100-104). */
int bem_boundary_matrix(const void* geom, int layer, int order, float k, const float* normals,
                        const float* curls, void* out, bem_stream_t stream);

/* Fused single-layer + double-layer assembly (exact order): one pass over
 * all triangle pairs evaluates each distance and phase once for both.
 *   v_out (may be NULL)  <- V
 *   k_out (may be NULL)  <- mass_coeff * M + k_coeff * K
 * With mass_coeff = 0.5, k_coeff = -1 this is the CBIE left-hand side
 * 0.5 I - K of src/bem/solver.py:97-104. */
int bem_boundary_matrices_vk(const void* geom, float k, void* v_out, void* k_out, float mass_coeff,
                             float k_coeff, bem_stream_t stream);

/* Batched fused assembly: many problems (meshes of any size, each with its
 * own wavenumber) in one persistent launch whose CTAs drain a single queue of
 * (problem, 32 test triangles, trial-tile chunk) work items, plus one launch
 * per touching-pair type over all problems.  `problems` is a HOST array;
 * every v_out / k_out must be non-NULL (nv x nv complex64, overwritten with V
 * and mass_coeff M + k_coeff K).  Workspace: bem_batch_workspace_bytes.
 * No counterpart in the reference (one mesh, one wavenumber per call). */
typedef struct bem_batch_problem {
  const void* geom; /* built geometry */
  float k;          /* wavenumber */
  void* v_out;
  void* k_out;
} bem_batch_problem;
size_t bem_batch_workspace_bytes(int nproblems);
int bem_batch_matrices_vk(const bem_batch_problem* problems, int nproblems, float mass_coeff, float k_coeff,
                          void* workspace, size_t workspace_bytes, bem_stream_t stream);

/* Fused Burton-Miller assembly: both matrices of a Burton-Miller system
 * with coupling i/k in one pass, at quadrature `order`,
 *   lhs_out <- bm_lhs_boundary_matrix[order] + 1/2 M
 *   rhs_out <- bm_rhs_boundary_matrix[order] - (i / (2k)) M
 * (both required, nv x nv complex64, overwritten; k != 0).  With
 * BEM_ORDER_APPROX these are BEM_Solver.neumann2dirichlet's matrices
 * (src/bem/solver.py:118-126: the bindings bind.cu:204-215, identity_matrix
 * and the elementwise combination done in Python); with BEM_ORDER_EXACT they
 * equal BEM_Solver.HBIE's (solver.py:106-116): 1/2 M - K + (i/k) W and
 * -V - (i/k)(K' + 1/2 M). */
int bem_boundary_matrices_bm(const void* geom, int order, float k, void* lhs_out, void* rhs_out,
                             bem_stream_t stream);

/* Batched fused Burton-Miller assembly (one persistent launch over all
 * problems' regular pairs, one launch per touching-pair type).  `problems`
 * is a HOST array.  Workspace: bem_batch_workspace_bytes (sized for both
 * batched assemblies).  No counterpart in the reference; its multi-mode
 * caller (src/scene.py:384-397) assembles one mode at a time. */
typedef struct bem_bm_problem {
  const void* geom; /* built geometry */
  float k;          /* wavenumber (!= 0) */
  void* lhs_out;
  void* rhs_out;
} bem_bm_problem;
int bem_batch_matrices_bm(const bem_bm_problem* problems, int nproblems, int order, void* workspace,
                          size_t workspace_bytes, bem_stream_t stream);

/* BEM_OK, or BEM_ERR_CUDA if a bounded wait of an assembly kernel (the bulk
 * copies of trial tiles) expired anywhere in this process since the last
 * call, on any stream and geometry; clears the process-wide flag and
 * synchronises `stream`.  bem_geometry_status reports the same per geometry.
 * No counterpart in the reference. */
int bem_assembly_status(bem_stream_t stream);

/* Launch-shape knobs of the assembly kernels, set by the autotuner
 * (0 = automatic).  Process-wide. */
enum {
  BEM_TUNE_ASSEMBLY_CHUNK = 1,      /* trial tiles (16 triangles) per work item */
  BEM_TUNE_ASSEMBLY_CTAS_PER_SM = 2, /* persistent CTAs per SM (<= occupancy limit) */
  BEM_TUNE_TC_PROMOTE = 3,           /* tensor-core matvec: K blocks (64 reals) accumulated in tensor
                                        memory before the partial sum leaves it (0: automatic) */
  BEM_TUNE_GMRES_REORTH = 4,         /* Arnoldi Gram-Schmidt passes: 0 automatic (one), 1 one, 2 two */
  BEM_TUNE_ARNOLDI_CLUSTER = 5,      /* largest thread-block cluster (<= 16 CTAs) per Krylov column in
                                        the Arnoldi kernel (0: automatic) */
  BEM_TUNE_ARNOLDI_MODE = 6,         /* Arnoldi step: 0 automatic (1), 1 one cluster kernel per step,
                                        2 streamed kernels over all SMs, 3 one cooperative kernel over
                                        all SMs (two grid barriers; falls back to 1 when its grid does
                                        not fit) */
  BEM_TUNE_TC_WAIT_US = 7,           /* limit of each bounded wait in the tensor-core matvec, microseconds
                                        (0: 2 s) */
  BEM_TUNE_TC_TEST_SKIP_FILL = 8,    /* test hook for the bounded waits, one launch: value v > 0 makes CTA 0
                                        of the next tensor-core matvec leave its (v-1)-th pipeline fill
                                        unissued, so the consumer's wait expires, the kernel drains its
                                        copies and returns, and bem_tc_status reports BEM_ERR_CUDA
                                        (no fault, no hang); 0 = off */
  BEM_TUNE_GMRES_BLOCK = 9           /* bem_gmres_solve with 2..64 right-hand sides: 0 block GMRES (the
                                        default; one block Krylov space per group of <= 16 columns, the
                                        groups sharing each matvec), 1 one space per column */
};
int bem_set_tuning(int key, int value);
int bem_get_tuning(int key);

/* Dense P1 mass matrix (bind.cu:10-21), overwriting out. */
int bem_identity_matrix(const void* geom, void* out, bem_stream_t stream);

/* Per-triangle complex values averaged onto vertices, bind.cu:23-48.
 * tri_values (nt) complex64 -> out (nv) complex64.  `counts` is an int32
 * scratch array of nv entries. */
int bem_triangle2vertex(const void* geom, const void* tri_values, void* out, int* counts,
                        bem_stream_t stream);

/* Listener potential matrix (np x nv complex64, overwritten) of the single
 * (layer 0) or double (layer 1) layer, bind.cu:156-176. */
int bem_potential_matrix(const void* geom, int layer, const float* points, int np, float k, void* out,
                         bem_stream_t stream);

/* Fused listener evaluation without a potential matrix:
 *   out(:, s) = -S neumann(:, s) + D dirichlet(:, s),   s = 0..nrhs-1
 * (src/bem/solver.py:140-147).  neumann/dirichlet are (nv, nrhs) complex64
 * row-major (either may be NULL = zero); out is (np, nrhs) complex64,
 * overwritten.  scratch: bem_boundary2potential_scratch_bytes() bytes. */
size_t bem_boundary2potential_scratch_bytes(int nt, int nrhs);
int bem_boundary2potential(const void* geom, const float* points, int np, float k, const void* neumann,
                           const void* dirichlet, int nrhs, void* out, void* scratch,
                           size_t scratch_bytes, bem_stream_t stream);

/* Listener evaluation for callers that cannot allocate device memory (for
 * example a real-time audio or rendering loop, where an allocation may block
 * and synchronise the device past the callback deadline, or a C plug-in with
 * no device allocator of its own).  Same result as bem_boundary2potential, no
 * scratch argument: the densities live in a fixed 16 MiB array of the
 * library's own device memory, reserved on every GPU that loads the library.
 * Limit: 6 * nt * nrhs <= bem_boundary2potential_noalloc_max() (2^20), else
 * BEM_ERR_WORKSPACE before any work.  The first call on a device (with it
 * current) looks up the array's address; make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Calls no cudaMalloc/cudaFree.
 * No counterpart in the reference, which allocates its outputs with torch. */
long long bem_boundary2potential_noalloc_max(void);
int bem_boundary2potential_noalloc(const void* geom, const float* points, int np, float k, const void* neumann,
                                   const void* dirichlet, int nrhs, void* out, bem_stream_t stream);

/* ------------------------------------------------------------------------
 * Dense complex linear algebra.
 * ---------------------------------------------------------------------- */

/* Y = A X for an n x n complex64 row-major A and m right-hand sides
 * X (n, m) row-major complex64 -> Y (n, m) complex64 (overwritten).
 * Replaces the cuBLAS gemv the reference calls through torch `@`
 * (src/bem/solver.py:103,147; BiCGSTAB.py:52,68,73). */
int bem_cmatmul(const void* A, int n, const void* X, int m, void* Y, bem_stream_t stream);

/* ------------------------------------------------------------------------
 * Adjoint (differentiation).  No counterpart in the reference, which has no
 * gradients; these serve the hand-written adjoint of the listener pressures
 * p = -S g + D u, (1/2 M - K) u = -V g.
 * ---------------------------------------------------------------------- */

/* Y = A^H X for an n x n complex64 A and m columns (Y overwritten). */
int bem_cmatmul_adjoint(const void* A, int n, const void* X, int m, void* Y, bem_stream_t stream);
/* out = conj(A)^T (n x n complex64, out != A). */
int bem_conj_transpose(const void* A, int n, void* out, bem_stream_t stream);
/* out_s = S^H pbar, out_d = D^H pbar (each nv complex64, either may be NULL)
 * for np listener weights pbar (complex64). */
int bem_boundary2potential_adjoint(const void* geom, const float* points, int np, float k, const void* pbar,
                                   void* out_s, void* out_d, bem_stream_t stream);
/* grad (nv x 3 float64, overwritten) = d/dx Re[ -pbar^H S g + pbar^H D u
 *   - lambda^H V g - 1/2 lambda^H M u + lambda^H K u ] with the vectors held
 * fixed (lambda, g = neumann, u = dirichlet: nv complex64; pbar: np). */
int bem_vertex_gradient(const void* geom, float k, const void* lambda, const void* neumann, const void* dirichlet,
                        const float* points, int np, const void* pbar, double* grad, bem_stream_t stream);

/* Solver precision of the dense operator. */
enum {
  BEM_PREC_FP32 = 0,   /* complex64 CUDA-core matvec */
  BEM_PREC_BF16X3 = 1, /* tensor-core bf16 hi/lo split (3 products), FP32 accumulate */
  BEM_PREC_BF16 = 2,   /* tensor-core bf16 (1 product), FP32 accumulate */
  BEM_PREC_FP16X3 = 3  /* tensor-core fp16 hi/lo split with power-of-two row / column scales
                          (3 products): FP32-level accuracy at the bytes of BF16X3 */
};

typedef struct bem_solver_params {
  int precision;     /* BEM_PREC_* of the inner Krylov matvec */
  int restart;       /* GMRES restart length (Krylov dimension), >= 1 */
  int max_iters;     /* total inner iterations per solve */
  int max_refine;    /* outer FP64 refinement steps (>= 1) */
  double rtol;       /* stop when ||b - A x|| <= rtol ||b|| (per column) */
  double atol;       /* or when ||b - A x|| <= atol */
  double inner_rtol; /* inner GMRES tolerance relative to its own RHS */
} bem_solver_params;

typedef struct bem_solver_info {
  int status;         /* bem_status of the whole solve */
  int iterations;     /* inner iterations (max over columns) */
  int refinements;    /* outer refinement steps taken */
  int matvecs;        /* operator applications */
  double rel_residual; /* max over columns of ||b - A x|| / ||b|| (FP64, FP32 A) */
} bem_solver_info;

/* Tensor-core operator (tcgen05): the complex64 matrix A is split into bf16
 * planes once (bem_tc_operator_prepare), after which bem_tc_matmul computes
 * Y = A X for m <= 128 right-hand sides with FP32 accumulation in tensor
 * memory.  precision: BEM_PREC_BF16X3 (A and X split hi/lo, three products)
 * BEM_PREC_BF16 (A in bf16, X split, two products) or BEM_PREC_FP16X3 (fp16
 * hi/lo splits with power-of-two scales, three products).  No counterpart in the
 * reference (it multiplies with cuBLAS through torch). */
size_t bem_tc_operator_bytes(int n, int m, int precision);
int bem_tc_operator_prepare(const void* A, int n, int precision, void* workspace, size_t workspace_bytes,
                            bem_stream_t stream);
int bem_tc_matmul(const void* workspace, size_t workspace_bytes, int n, int precision, const void* X, int m,
                  void* Y, bem_stream_t stream);
/* BEM_OK, or BEM_ERR_CUDA if a tensor-core kernel on this workspace gave up
 * a bounded wait since the last call (its output is then not usable);
 * clears the flag and synchronises `stream`. */
int bem_tc_status(const void* workspace, bem_stream_t stream);

/* Workspace bytes for bem_gmres_solve (n unknowns, m right-hand sides). */
size_t bem_gmres_workspace_bytes(int n, int m, const bem_solver_params* params);

/* Solve A X = B for m right-hand sides with restarted GMRES wrapped in FP64
 * iterative refinement against the FP32 matrix.  2..64 right-hand sides: block
 * GMRES (block Krylov spaces of <= 16 columns, FP64 block Gram-Schmidt and
 * CholQR on the device, the small least-squares problems on the host);
 * otherwise one Krylov space per column (device-resident Arnoldi, FP64
 * classical Gram-Schmidt, Givens rotations).
 * A: n x n complex64 row-major.  B: (n, m) complex64.  X: (n, m) complex64,
 * used as the initial guess when `use_x0` != 0 and overwritten with the
 * solution.  `info` is a HOST pointer.  Synchronises `stream` once per
 * restart cycle.  Replaces solve_linear_equation / BiCGSTAB
 * (src/bem/solver.py:61-66, src/bem/BiCGSTAB.py:5-107). */
int bem_gmres_solve(const void* A, int n, const void* B, int m, void* X, int use_x0,
                    const bem_solver_params* params, void* workspace, size_t workspace_bytes,
                    bem_solver_info* info, bem_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* BEM_B200_H */
