/*
 * cfd_b200.h — C ABI of the B200 (sm_100a) kernels for the degree-4 nodal DG
 * Euler hot path of CFD-demo.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), returns 0 on success or a negative CFD_E* code, never
 * allocates device memory, and never synchronises the stream. The message of
 * the last failure on the calling thread is in cfd_last_error().
 *
 * Device state layout ("element-major SoA"): a state with K elements is an
 * array q[(c * 15 + j) * ld + e] for conserved variable c in (rho, rho u,
 * rho v, E), node j in 0..14 (the reference triangle's node order) and element
 * e in 0..K-1, with ld >= K. The reference's host layout (Np, K, 4) is
 * converted by cfd_pack_state / cfd_unpack_state. Precision CFD_FP64 stores
 * doubles; CFD_FP32_MIXED stores floats (averages, positivity pressure
 * recovery and all global reductions stay in double).
 *
 * Reference interfaces replaced (paths relative to the CFD-demo project):
 *   cfd_rhs            src/cfd_demo/dg.py:140-165          dg_rhs
 *   cfd_limit          src/cfd_demo/limiting.py:203-216    apply_limiters
 *   cfd_time_step      src/cfd_demo/time_integration.py:37-41  stable_time_step
 *   cfd_rk3_attempt    src/cfd_demo/time_integration.py:44-84  ssp_rk3_step
 *   cfd_run_control    src/cfd_demo/solver.py:167-216       EulerSolver.run loop body
 *   cfd_cell_averages  src/cfd_demo/dg.py:168-171          cell_averages
 *   cfd_integrate      src/cfd_demo/dg.py:174-176          domain_integral
 *   cfd_check_state    src/cfd_demo/solver.py:170-176      initial admissibility
 *   cfd_interface_flux src/cfd_demo/fluxes.py:28-159       rusanov / roe / hllc
 *   cfd_limiter_phi    src/cfd_demo/limiters.py:16-57      phi(r)
 *   cfd_mesh_build     src/cfd_demo/mesh.py:135-291, limiting.py:51-94  connectivity,
 *                      geometry, Cockburn-Shu coefficients, face-node pairing
 */
#ifndef CFD_B200_H
#define CFD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFD_ABI_VERSION 2

/* error codes */
#define CFD_OK 0
#define CFD_E_ARG (-1)     /* invalid argument (null pointer, bad id, bad size) */
#define CFD_E_CUDA (-2)    /* a CUDA launch or API call failed */

/* interface flux ids (fluxes.py:146-150) */
#define CFD_FLUX_RUSANOV 0
#define CFD_FLUX_ROE 1
#define CFD_FLUX_HLLC 2

/* limiter ids (limiters.py:42-48) */
#define CFD_LIMITER_MINMOD 0
#define CFD_LIMITER_MC 1
#define CFD_LIMITER_VAN_LEER 2
#define CFD_LIMITER_SUPERBEE 3
#define CFD_LIMITER_UNLIMITED 4

/* precision ids */
#define CFD_FP64 0
#define CFD_FP32_MIXED 1

/* boundary kinds (boundary.py:13-14); 0 = interior face */
#define CFD_FACE_INTERIOR 0
#define CFD_FACE_SLIP_WALL 1
#define CFD_FACE_FIXED_STATE 2
#define CFD_FACE_EXACT_STATE 3

/* entries of CfdSolver.limit_list ahead of its element list (counters) */
#define CFD_LIMIT_LIST_HEADER 16

/* run status (CfdControl.status) */
#define CFD_RUN_ACTIVE 0
#define CFD_RUN_DONE 1
#define CFD_RUN_BAD_DT (-1)
#define CFD_RUN_REJECTED (-2)

/*
 * Mesh tables in device memory, one entry per element unless stated; every
 * per-element array has leading dimension ld. Several instances (meshes) may
 * be concatenated: element e belongs to instance instance[e] (NULL: one
 * instance), and neighbour indices are global element indices.
 *
 * face_info[e] packs, for face f = 0, 1, 2, the 8-bit field
 * (face_info >> 8 f) & 0xff =
 *     kind (bits 0-1, CFD_FACE_*) | neighbour's local face (bits 2-3)
 *   | Cockburn-Shu partner face (bits 4-5) | reserved (bits 6-7).
 * Face node k of face f meets node 4-k of the neighbour's face g when f and g
 * are both 2 or both not 2, and node k otherwise (the face-2 nodes run against
 * the counterclockwise direction); the host checks this rule by coordinates.
 * neighbor[f * ld + e] is the neighbour element across face f for interior
 * faces and, for fixed-state faces, the row of bc_states (4 doubles) holding
 * the exterior state. For exact-state faces (CFD_FACE_EXACT_STATE: exterior
 * states from a known solution, one per face node) it is the first of 6
 * rows: the exterior states at the face's 5 nodes in this element's
 * face-node order, then the ghost cell average the troubled-cell test uses
 * across the face.
 */
typedef struct CfdMesh {
    int32_t num_elements;  /* K: elements of all instances */
    int32_t ld;            /* leading dimension, >= num_elements */
    int32_t num_instances; /* >= 1 */
    int32_t flags;         /* bit 0: every instance starts at a multiple of 64 elements
                              (padding elements have instance -1); required by the tiled
                              stage kernels when num_instances > 1 */
    const double* metric;    /* [4][ld]  rx, ry, sx, sy */
    const double* face_geo;  /* [9][ld]  nx_f, ny_f, Fscale_f (= sJ/J) for f = 0,1,2 */
    const double* face_hlen; /* [3][ld]  half edge length (boundary-flux weights) */
    const double* dt_geo;    /* [ld]     min_e 2|K| / ((N+1)^2 |e|) */
    const double* jacobian;  /* [ld]     J = |K| / 2 */
    const double* cs_coef;   /* [6][ld]  alpha_f, beta_f (limiting.py:51-94) */
    const int32_t* neighbor; /* [3][ld] */
    const int32_t* face_info;/* [ld] */
    const int32_t* instance; /* [ld] instance of each element, or NULL */
    const double* bc_states; /* [rows][4] fixed exterior states */
    const float* metric32;   /* FP32 copies for CFD_FP32_MIXED, else NULL */
    const float* face_geo32;
    const float* cs_coef32;
} CfdMesh;

/*
 * Input of cfd_mesh_build (device arrays): one mesh and its boundary tags.
 * The tag tables give, per tag index, the boundary kind and, for fixed-state
 * tags, the row of bc_states holding the exterior state.
 */
typedef struct CfdMeshBuild {
    int32_t num_vertices;
    int32_t num_elements;          /* K */
    int32_t ld;                    /* leading dimension of the output tables, >= K */
    int32_t num_boundary_edges;
    int32_t num_tags;
    int32_t reserved;
    const double* vertices;        /* [Nv][2] */
    const int64_t* elements;       /* [K][3] counterclockwise vertex ids, each < num_vertices */
    const int64_t* boundary_edges; /* [nb][2] vertex ids of every tagged boundary edge */
    const int32_t* boundary_tag;   /* [nb] tag index of each edge */
    const int32_t* tag_kind;       /* [tags] CFD_FACE_SLIP_WALL | CFD_FACE_FIXED_STATE (exact-state
                                      tags need per-node rows: build those tables on the host) */
    const int32_t* tag_row;        /* [tags] bc_states row of a fixed-state tag */
} CfdMeshBuild;

/* status bits of cfd_mesh_build */
#define CFD_SETUP_NONCONFORMING 1         /* a face shared by more than two elements */
#define CFD_SETUP_DOUBLE_TAG 2            /* a boundary edge with more than one tag */
#define CFD_SETUP_UNTAGGED 4              /* a boundary face without a tag */
#define CFD_SETUP_TAG_NOT_BOUNDARY 8      /* a tagged edge that is not a boundary face */
#define CFD_SETUP_NO_COEFFICIENTS 16      /* no nonnegative Cockburn-Shu coefficients */
#define CFD_SETUP_NOT_CONFORMING_NODES 32 /* neighbouring face nodes do not coincide */
#define CFD_SETUP_TABLE_FULL 64           /* internal hash table full (not expected) */
#define CFD_SETUP_UNSUPPORTED_KIND 128    /* a tag of another kind than slip wall / fixed state */

/* Per instance and per RK stage reduction slots (zeroed by cfd_rk3_attempt). */
typedef struct CfdStageAcc {
    double boundary_flux[4];        /* sum of w * sJ * Fhat over boundary face nodes */
    unsigned long long min_rho_key; /* ordered key of the minimum nodal density */
    unsigned long long min_p_key;   /* ordered key of the minimum nodal pressure */
    unsigned long long dt_key;      /* ordered key of min_K dt_geo / lambda_K (stage 3) */
    int32_t troubled;               /* troubled-cell count */
    int32_t flags;                  /* bit 0: non-finite value; bit 1: average rho or p <= 0 */
} CfdStageAcc;

/* StepReport of time_integration.py:22-29 (written by cfd_rk3_attempt). */
typedef struct CfdStepReport {
    double boundary_flux[4]; /* dt (B0/6 + B1/6 + 2 B2/3) */
    double min_density;
    double min_pressure;
    double dt;               /* the step size used */
    double dt_next;          /* CFL step of the new state (time_step(q_new)) */
    int32_t admissible;
    int32_t troubled_cells;
    int32_t reserved[2];
} CfdStepReport;

/* Host run-loop state of solver.py:177-204, kept on the device per instance. */
typedef struct CfdControl {
    double time;
    double final_time;
    double dt;            /* step size of the current attempt */
    double flux_integral[4];
    double min_density;
    double min_pressure;
    int32_t steps;
    int32_t rejected;
    int32_t attempts;     /* failed attempts of the current step */
    int32_t max_troubled;
    int32_t parity;       /* which of (x0, x1) holds the current state */
    int32_t status;       /* CFD_RUN_* */
    int32_t reaches_end;
    int32_t reserved;
} CfdControl;

/* Solver description: mesh + configuration + caller-owned scratch. */
typedef struct CfdSolver {
    CfdMesh mesh;
    int32_t flux;          /* CFD_FLUX_* */
    int32_t limiter;       /* CFD_LIMITER_* */
    int32_t precision;     /* CFD_FP64 | CFD_FP32_MIXED */
    int32_t max_rejections;
    double gamma;
    double cfl;
    /* scratch, caller-allocated device memory */
    double* averages;      /* [4][ld] stage cell averages (double in both precisions) */
    double* element_aux;   /* [3][ld] per-element min rho, min p, lambda (limited runs) */
    CfdStageAcc* acc;      /* [num_instances][3] */
    CfdStepReport* report; /* [num_instances] */
    CfdControl* control;   /* [num_instances] */
    int32_t block_size;    /* threads per block of the pair stage kernel (64, 128, 256); 0 = default */
    int32_t variant;       /* stage kernel: 0 tiled (default), 1 tiled + staged base rows,
                              2 register-only pair kernel, 3 tiled with 64 elements per block,
                              4 tiled with registers capped for more resident blocks,
                              5 tiled with 64 elements per block and the face rounds kept rolled,
                              6 / 7 as 3 / 5 with scalar FMAs in the FP32 [Dr|Ds] and LIFT
                              contractions, which the other tiled shapes issue as packed
                              FP32x2 FMAs (bitwise the same results; FP64 runs 3 / 5),
                              8 tiled with 64 elements per block + staged base rows,
                              9 as 8 with the face-node flux as an out-of-line call (FP32),
                              10 / 11 the face-job form of 3 / 8: each face's flux is evaluated
                              once, by the block's owner of the face, for both of its sides,
                              12 / 13 as 9 with the volume node loop kept rolled ([Dr|Ds] from
                              the constant bank), with unrolled / rolled face rounds,
                              14 as 5 with the volume node loop kept rolled */
    int32_t* limit_list;   /* optional [CFD_LIMIT_LIST_HEADER + ld] scratch: with it the limiter
                              runs in two passes (a light detection pass over every element,
                              then the rewrite of the troubled / non-positive ones only);
                              NULL: one pass. cfd_rk3_begin resets its counters. */
    uint8_t* troubled_flags; /* optional [3][ld]: the troubled-cell indicator of limiting.py:147-151
                              (1 = troubled, 0 = not) of every active element; stage k of an attempt
                              writes row k-1, cfd_limit writes row 0. NULL: not written. */
} CfdSolver;

/* ---- library ------------------------------------------------------------- */
int cfd_abi_version(void);
/* sizeof CfdMesh, CfdStageAcc, CfdStepReport, CfdControl, CfdSolver (host only;
 * lets a binding check its struct layouts). */
int cfd_struct_sizes(int32_t* out, int32_t n);
const char* cfd_last_error(void);

/* Layout conversion: host layout (Np, K, 4) double <-> device layout of
 * `precision`. Both pointers are device memory. */
int cfd_pack_state(const double* q_nk4, void* q_dev, int32_t K, int32_t ld, int32_t precision, void* stream);
int cfd_unpack_state(const void* q_dev, double* q_nk4, int32_t K, int32_t ld, int32_t precision, void* stream);

/* ---- operators (one instance or all instances at once) --------------------
 * cfd_rhs: rhs = L(q) (dg.py:140-165) and, per instance, the boundary flux
 * integral bflux[inst*4 + c] (zeroed by the call). */
int cfd_rhs(const CfdSolver* s, const void* q, void* rhs, double* bflux, void* stream);

/* cfd_limit: apply_limiters (limiting.py:203-216) from q_in to q_out (may
 * alias); troubled[inst] receives the troubled-cell count. */
int cfd_limit(const CfdSolver* s, const void* q_in, void* q_out, int32_t* troubled, void* stream);

/* cfd_time_step: dt[inst] = cfl * min_K dt_geo / max_nodes(|u| + c). */
int cfd_time_step(const CfdSolver* s, const void* q, double* dt, void* stream);

/* cfd_cell_averages: avg[c * ld + e] (double); cfd_integrate: integral[inst*4 + c]. */
int cfd_cell_averages(const CfdSolver* s, const void* q, double* avg, void* stream);
int cfd_integrate(const CfdSolver* s, const void* q, double* integral, void* stream);

/* cfd_check_state: out[inst*3 + {0,1,2}] = min nodal density, min nodal
 * pressure, 1.0 if every value is finite else 0.0. */
int cfd_check_state(const CfdSolver* s, const void* q, double* out, void* stream);

/*
 * cfd_rk3_attempt: one SSP-RK3 step attempt (time_integration.py:44-84) for
 * every active instance. The current state of instance i is x0 if
 * control[i].parity == 0 else x1; the new state goes to the other buffer;
 * stage is a third state buffer. dt is control[i].dt. Writes report[i]
 * (including dt_next, the CFL step of the new state). Instances whose
 * control.status != CFD_RUN_ACTIVE are skipped. The parity is NOT flipped:
 * cfd_run_control (or the caller) accepts the step.
 */
int cfd_rk3_attempt(const CfdSolver* s, void* x0, void* x1, void* stage, void* stream);

/* The three parts of cfd_rk3_attempt, for callers that interleave their own
 * work or timing: begin zeroes the reduction slots; stage k (1, 2, 3) runs
 * the fused DG stage kernel and, unless the limiter is `unlimited`, the
 * limiter kernel; finish writes the report. */
int cfd_rk3_begin(const CfdSolver* s, void* stream);
int cfd_rk3_stage(const CfdSolver* s, void* x0, void* x1, void* stage, int32_t k, void* stream);
int cfd_rk3_finish(const CfdSolver* s, void* stream);

/*
 * cfd_run_control: the body of the reference's run loop (solver.py:180-204)
 * after an attempt, per instance: accept (flip parity, advance time, count,
 * accumulate boundary flux and minima, take dt_next clipped to the final
 * time) or reject (halve dt, up to max_rejections), setting status to DONE or
 * an error when the loop would end.
 */
int cfd_run_control(const CfdSolver* s, void* stream);

/*
 * cfd_batch_advance: `attempts` passes of (cfd_rk3_attempt + cfd_run_control)
 * for every instance in ONE persistent, cooperative launch (no counterpart in
 * the reference, which solves one problem per EulerSolver; this is the
 * batched form of its run loop, solver.py:180-204). The grid holds as many
 * blocks as are resident on the GPU at once (or one per element tile of 64
 * elements, if there are fewer tiles); they loop over the element
 * tiles of all instances, with a grid-wide barrier between the phases of an
 * attempt (zero the reduction slots; stage k and its limiter passes for
 * k = 1, 2, 3; report and control). Returns early once no instance is active.
 * Needs the limit_list scratch (the limiter runs in its two-pass form). The
 * tile shape is fixed per precision (FP32: variant 9, FP64: variant 3) and the
 * per-element arithmetic is that of the separate launches, so the results
 * equal those of `attempts` x (cfd_rk3_attempt + cfd_run_control) with that
 * variant: bit for bit in FP32-mixed, to the last bits in FP64 (where the
 * compiler may contract a multiply-add differently in the two kernels).
 * The first call on a device looks up the resident grid size: make it before
 * any stream capture (a call with attempts = 0 does only that).
 */
int cfd_batch_advance(const CfdSolver* s, void* x0, void* x1, void* stage, int32_t attempts, void* stream);

/* cfd_run_init: control[i] = {time 0, final_time[i], dt = clipped CFL step of
 * the current state, ...}; minima start from the nodal minima of the state. */
int cfd_run_init(const CfdSolver* s, const void* x0, const double* final_time, void* stream);

/*
 * cfd_rk3_step_noalloc: one SSP-RK3 step of one mesh at the given dt, from
 * q_in to q_out (device layout, leading dimension mesh->ld), writing the step
 * report to the device pointer `report`. It has no counterpart in the
 * reference. It is for callers that cannot allocate device memory: a
 * foreign-language binding that holds only the buffers it was handed and has
 * no CUDA allocator of its own, or an application whose memory pool forbids
 * outside allocations once it runs. Every scratch buffer of the step lives in
 * a static device array inside this library, sized for meshes with
 * ld <= CFD_NOALLOC_MAX_ELEMENTS (about 9 MB, held on every GPU that loads the
 * library until the process exits); larger meshes are refused with CFD_E_ARG.
 * The call allocates nothing. Its first call on a device looks up the device
 * address of that array (cudaGetSymbolAddress), so make that first call
 * before any stream capture; first calls from several host threads at once
 * are safe (the lookup is done under a lock). The address stays cached for the
 * life of the process, so do not call this entry point on a device after a
 * cudaDeviceReset of that device. All calls share the one array: calls that
 * overlap on the GPU (other streams, other host threads) race, and the caller
 * must serialise them.
 */
#define CFD_NOALLOC_MAX_ELEMENTS 16384
int cfd_rk3_step_noalloc(const CfdMesh* mesh, int32_t flux, int32_t limiter, int32_t precision, double gamma,
                         double cfl, const void* q_in, void* q_out, double dt, CfdStepReport* report, void* stream);

/*
 * ---- discrete adjoint of the fixed-size RK3 step
 * The reference differentiates its step with jax.grad (fluxes.py:7 and
 * limiters.py:4 keep the code differentiable; solver.py:181 turns dt into a
 * host float, so dt is a constant of each step). These entries are its
 * hand-written replacement for EulerSolver._step (time_integration.py:44-84)
 * and its vector-Jacobian product; neither has a C counterpart in the
 * reference.
 *
 * cfd_rk3_step_fixed: one SSP-RK3 step of size dt[instance] (device array)
 * from q_in to q_out without CFL control or rejection; `stage` is scratch of
 * one state. The step report is left in s->report. When `tape` is not NULL it
 * receives what the adjoint needs (cfd_tape_bytes(ld, precision) bytes): the
 * stage states before and after limiting, the stage averages and minima, and
 * the positivity limiter's pressure-scaling theta; the stage kernels write it
 * as they go (the averages and minima go to the tape instead of
 * s->averages / s->element_aux).
 * The limiter of every configuration runs in its own kernel here, so the
 * result can differ in the last bits from cfd_rk3_attempt's fused positivity
 * for `unlimited`.
 *
 * cfd_rk3_step_adjoint: given the adjoint g_out of q_out, writes the adjoint
 * g_in of q_in (g_in = (dq_out/dq_in)^T g_out) for the step that produced
 * `tape` from q_in with the same dt, and adds the adjoint of the fixed
 * exterior states to bc_bar[rows][4] when bc_bar is not NULL (the caller
 * zeroes it). The limiter branches are those the forward step took. The
 * pressure-scaling theta of the positivity limiter (a bisection root) is
 * differentiated implicitly, as a finite difference of the step sees it; with
 * CFD_ADJ_HOLD_THETA in `flags` it is held constant instead, the derivative
 * jax.grad takes of the bisection loop. `work` is scratch of
 * cfd_adjoint_work_bytes(ld, precision) bytes.
 */
#define CFD_ADJ_HOLD_THETA 1
int64_t cfd_tape_bytes(int32_t ld, int32_t precision);
int64_t cfd_adjoint_work_bytes(int32_t ld, int32_t precision);
int cfd_rk3_step_fixed(const CfdSolver* s, const void* q_in, void* q_out, void* stage, const double* dt, void* tape,
                       void* stream);
int cfd_rk3_step_adjoint(const CfdSolver* s, const void* q_in, const void* tape, const double* dt, const void* g_out,
                         void* g_in, double* bc_bar, int32_t flags, void* work, void* stream);

/*
 * ---- mesh tables on the GPU
 * cfd_mesh_build: the mesh tables of `out` (metric, face_geo, face_hlen,
 * dt_geo, jacobian, cs_coef, neighbor, face_info; out->ld == in->ld and
 * out->num_elements == in->num_elements; the pointers must be writable device
 * memory) from the vertex and element arrays: geometry (mesh.py:216-243),
 * face connectivity and boundary tags (mesh.py:135-185), Cockburn-Shu
 * coefficients (limiting.py:51-94), every floating-point value bit for bit
 * the host builder's. face_node_bary: [3][5][3] barycentric weights of the
 * reference face nodes, for the check that face node k of face f meets node
 * k or 4 - k of the neighbour's face (mesh.py:254-291) within pairing_rtol of
 * the edge length. `work` is scratch of cfd_mesh_build_work_bytes bytes;
 * *status (device) receives CFD_SETUP_* bits describing an invalid input.
 */
int64_t cfd_mesh_build_work_bytes(int32_t num_elements, int32_t num_boundary_edges);
int cfd_mesh_build(const CfdMeshBuild* in, const CfdMesh* out, const double* face_node_bary, double pairing_rtol,
                   void* work, int64_t work_bytes, int32_t* status, void* stream);

/* ---- pointwise physics (exercise the device functions of the fused kernels) */
int cfd_interface_flux(int32_t flux, int32_t n, const double* q_minus, const double* q_plus,
                       const double* nx, const double* ny, double gamma, double* out, void* stream);
int cfd_limiter_phi(int32_t limiter, int32_t n, const double* r, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CFD_B200_H */
