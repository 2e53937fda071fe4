/*
 * dgb200 -- B200 (sm_100a) hybrid-mesh DG residual-and-update path, C ABI.
 *
 * Drop-in boundary for the Python entry points of superboss2300/jax-fluid-sim
 * (a pure Python/JAX project: there is no FFI in the reference; each entry
 * point below names the Python method whose behaviour it replaces).
 *
 * Conventions
 *   - All state arrays are DEVICE pointers owned by the caller, one per element
 *     block in the reference's block order (hexahedron, wedge, tetra), each a
 *     contiguous float64 array (elements, nodes, variables) -- the reference's
 *     state layout (hybrid/state.py:7-37, hybrid/mesh.py:253-286).
 *   - Plan tables are HOST pointers; dgb_plan_* copies them to the device and
 *     the plan owns the copies.
 *   - Return 0 on success, a negative dgb_error code on failure; the message of
 *     the last failure on this thread is in dgb_last_error().
 *   - A plan is not thread-safe; every call takes the CUDA stream to run on.
 */
#ifndef DGB200_H
#define DGB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum dgb_error {
  DGB_OK = 0,
  DGB_ERR_ARGUMENT = -1,   /* invalid argument or plan state (reference raises ValueError) */
  DGB_ERR_CUDA = -2,       /* CUDA runtime failure */
  DGB_ERR_UNSUPPORTED = -3 /* configuration outside what the kernels implement */
};

enum { DGB_MAX_BLOCKS = 3, DGB_MAX_TAGS = 8, DGB_MAX_VARS = 16 };

typedef struct dgb_plan dgb_plan;

/* Physics, boundary and limiter constants.
 *   HybridCompressibleSolver.__init__   hybrid/solver.py:20-61
 *   FarfieldWallBoundary.__init__        hybrid/boundary.py:13-46
 *   HybridPositivityLimiter.__init__     hybrid/limiter.py:14-26
 *   HybridSSPRK3.__init__                hybrid/time_integration.py:9-25
 *   HybridTroubledCellSensor.__init__    hybrid/limiter.py:153-163 */
typedef struct {
  int degree;                 /* 1..3 */
  int nvars;                  /* 5 + species (5 or 16) */
  int num_blocks;             /* 1..3 */
  int viscous;                /* 1 when dynamic_viscosity > 0 */
  double gamma, gas_constant, dynamic_viscosity, thermal_conductivity, br2_penalty;
  int has_boundary;           /* 0: boundary_state=None (ghost = interior trace) */
  double farfield_primitive[DGB_MAX_VARS];
  int inlet_tags[DGB_MAX_TAGS], n_inlet;
  int wall_tags[DGB_MAX_TAGS], n_wall;
  int no_slip_tags[DGB_MAX_TAGS], n_no_slip;
  int slip_tags[DGB_MAX_TAGS], n_slip;
  int has_wall_temperature;
  double wall_temperature;
  double pos_density_floor, pos_pressure_floor, pos_relative_floor;
  double adm_density_floor, adm_pressure_floor;
  double sensor_threshold;
  int limiter;                /* stage limiter of dgb_ssprk3_step: 0 none, 1 positivity, 2 MOOD */
  int reconstruction;         /* MOOD subcell faces: 0 constant, 1 tvd, 2 weno (CWENO-Z) */
  int precision;              /* 0 float64 throughout; 1 mixed: float32 arithmetic and shared-memory
                                 staging in the trace, BR2-lift, volume and finalize kernels of
                                 every element type (state, face fluxes, limiters, reductions and
                                 the stage update stay float64) */
} dgb_params;

/* One element block (hybrid/geometry.py:139-203 metrics, precomputed by the host). */
typedef struct {
  int element_type;           /* 0 hexahedron, 1 wedge, 2 tetra */
  int num_elements, num_nodes, num_qp, num_local_faces;
  const double* basis;        /* [Nq][Np]      basis at volume points          */
  const double* basis_grad;   /* [Nq][Np][3]   reference gradients              */
  const double* inv_jacobian; /* [E][Nq][3][3] dxi_r/dx_d                       */
  const double* wdet;         /* [E][Nq]       w |det J|                        */
  const double* inv_mass;     /* [E][Np][Np]   sliver-scaled inverse mass; stored transposed
                                 ([E][j][i] = M^-1[i][j]) when dgb_plan_set_hex is used; may be
                                 NULL, then dgb_plan_build_inverse_mass forms it on the device */
  const int32_t* elem_face;   /* [E][nlf]      (face type<<30)|(face<<1)|side   */
  const double* length;       /* [E]           characteristic length (CFL)      */
  int num_face_samples;
  const double* face_sample_basis; /* [Ns][Np] basis at distinct face points    */
  const double* p1_projector;      /* [Np][Np] sensor projector (P>=2)          */
} dgb_block_desc;

/* One face type (hybrid/mesh.py:378-459 topology, hybrid/geometry.py:226-362 metrics). */
typedef struct {
  int face_type;              /* 0 triangle, 1 quad */
  int num_faces, num_qp;
  const int32_t* owner_block; const int32_t* owner_local; const int32_t* owner_code;
  const int32_t* nbr_block;   const int32_t* nbr_local;   const int32_t* nbr_code;  /* -1: boundary */
  const int32_t* tags;        /* physical tag, -1 internal */
  const double* normals;      /* [F][nq][3] */
  const double* weights;      /* [F][nq]    */
  const double* side_inv_jacobian; /* [F][2][nq][3][3] at owner / neighbour face points */
} dgb_face_desc;

/* Per-block device state pointers, (E_b, Np_b, nvars) float64 each. */
typedef struct {
  double* block[DGB_MAX_BLOCKS];
} dgb_state;

/* Admissibility of a stage/step (time_integration.py:291-312) in device memory. */
typedef struct {
  int32_t valid;
  int32_t pad;
  double rho_min;
  double p_min;
} dgb_status;

const char* dgb_last_error(void);
int dgb_version(void);

/* Plan lifetime. */
int dgb_plan_create(const dgb_params* params, dgb_plan** out);
int dgb_plan_set_block(dgb_plan* plan, int block, const dgb_block_desc* desc);
int dgb_plan_set_faces(dgb_plan* plan, const dgb_face_desc* desc);
/* Trace tables for (element type, face type): basis [C][nq][Np] and gradients [C][nq][Np][3]
 * at each code's reference face points. */
int dgb_plan_set_trace(dgb_plan* plan, int element_type, int face_type, int num_codes, int num_qp,
                       int num_nodes, const double* basis, const double* basis_grad);
/* Forms the sliver-scaled inverse mass matrices of block b on the device from the block's basis
 * and w|det J| tables, for a block whose descriptor gave inv_mass = NULL (hybrid/geometry.py:
 * 181-192 forms M = B^T diag(w|J|) B and inverts it on the host; the scale is
 * min(1, volume[e] / 1e-4)).  volume: host [E], the element volumes sum_q w|det J|.
 * transposed: store [E][j][i] (the layout of the sum-factorised path).  Synchronous (set-up);
 * fails on an element whose mass matrix is not positive definite. */
int dgb_plan_build_inverse_mass(dgb_plan* plan, int block, const double* volume, int transposed);
/* Set-up helper: inverts count symmetric positive definite n x n matrices (device memory,
 * [count][n][n], n <= 160) in place, one per CTA, by Gauss-Jordan elimination without pivoting;
 * *status (a device int) is set to 0, or to 1 + the index of a matrix found not positive
 * definite, which is then left partly reduced.  Asynchronous on stream.  Used for the
 * least-squares Gram matrices of the MOOD subcell reconstruction (hybrid/subcell.py:324-334
 * inverts them with a dense inverse). */
int dgb_spd_inverse(double* matrices, int n, int count, int* status, void* stream);
/* Host-side geometry metrics for plan set-up (no GPU needed; hybrid/geometry.py:139-203,
 * 299-353 form the same with dense einsums).  For count elements, element i taking the
 * geometry nodes nodes[index ? index[i] : i] ([n][3] each), at num_points reference points
 * with geometry-basis gradients grad[num_points][n][3]: jacobian [count][Q][3][3]
 * (J[d][r] = dx_d/dxi_r), det [count][Q], inv_jacobian [count][Q][3][3], wdet [count][Q]
 * = weights[q] |det J|; with tangents [Q][2][3] (reference face tangents t_u, t_v) and
 * orientation [count][3] (a direction the normal must not oppose): normals [count][Q][3]
 * (unit J t_u x J t_v) and area_weights [count][Q] = weights[q] |J t_u x J t_v|.  Any output
 * may be NULL.  Runs on the host cores in threads. */
int dgb_map_metrics(const double* nodes, const int32_t* index, int count, int num_nodes, const double* grad,
                    int num_points, const double* weights, const double* tangents, const double* orientation,
                    double* jacobian, double* det, double* inv_jacobian, double* wdet, double* normals,
                    double* area_weights);

/* (set-up, host threads, no GPU) Affine test of a block's per-point inverse Jacobians
 * jinv [count][num_points][9] (the isoparametric map is affine when J^-1 is the same at every
 * point): affine[e] = 1 when every entry equals the first point's to tol relative to the
 * element's largest |entry|; mean [count][9] the mean over the points.  Used to give affine
 * elements constant metrics and a tensor-product M^-1 (hybrid/geometry.py:181-192 forms the same
 * matrices by quadrature). */
int dgb_affine_test(const double* jinv, int count, int num_points, double tol, uint8_t* affine, double* mean);
/* Host-side subcell face metrics for the MOOD subcell plan (no GPU; hybrid/subcell.py:336-360).
 * For count elements with the physical subcell vertices vertices[count][num_vertices][3] and subcell
 * centres centers[count][num_subcells][3]: each face f of faces[num_faces][4] (face_sizes[f] = 3 or
 * 4 vertex ids) gets its area vector (a triangle p0 p1 p2: (p1 - p0) x (p2 - p0) / 2; a
 * quadrilateral adds (p2 - p0) x (p3 - p0) / 2), turned toward centre[neighbors[f]] -
 * centre[owners[f]] (or, with neighbors NULL, toward the face centre), as normals
 * [count][num_faces][3] (unit), areas [count][num_faces] and, when not NULL, face_centers
 * [count][num_faces][3] (the mean of the face's vertices).  Runs on the host cores in threads. */
int dgb_subcell_face_metrics(const double* vertices, int count, int num_vertices, const int32_t* faces,
                             const int32_t* face_sizes, int num_faces, const double* centers, int num_subcells,
                             const int32_t* owners, const int32_t* neighbors, double* normals, double* areas,
                             double* face_centers);

/* (set-up, host threads, no GPU) Face pairing of one face type (hybrid/mesh.py:378-459: every
 * (block, cell, local face) is visited in order and equal sorted corner keys are paired).  keys
 * [n][k] are the visits' sorted corner ids, visit [n] their distinct visiting order.  Writes the
 * faces in the reference's order, internal faces by their second visit and then boundary faces by
 * their first: owner[f] (the first visit's row), neighbor[f] (the second visit's row, -1 at the
 * boundary), *count faces (at most n).  A key visited more than twice is DGB_ERR_ARGUMENT with
 * the reference's message. */
int dgb_pair_faces(const int64_t* keys, int k, int64_t n, const int64_t* visit, int64_t* owner, int64_t* neighbor,
                   int64_t* count);
/* (set-up, host, no GPU) Numeric sections of Gmsh ASCII meshes (the reference reads them with
 * meshio, hybrid/mesh.py:182-236).  text/len: the section body after its "$Nodes" or "$Elements"
 * line.  MSH 2.2: dgb_msh2_nodes reads n records "id x y z" into ids [n], xyz [n][3];
 * dgb_msh2_elements reads n records "id type ntags tags... nodes..." into type [n], phys [n] (the
 * first tag, 0 without tags) and node ids nodes [cap] with offsets [n + 1].  MSH 4.1 (the body
 * starts with the section's count line): dgb_msh4_nodes reads the entity blocks' node tags and
 * coordinates (parametric coordinates skipped); dgb_msh4_elements gives each element its type,
 * its entity's dimension and tag, and its node ids.  Malformed records, counts that disagree with
 * the header and node lists beyond cap are DGB_ERR_ARGUMENT. */
int dgb_msh2_nodes(const char* text, int64_t len, int64_t n, int64_t* ids, double* xyz);
int dgb_msh2_elements(const char* text, int64_t len, int64_t n, int32_t* type, int32_t* phys, int64_t* offsets,
                      int64_t* nodes, int64_t cap);
int dgb_msh4_nodes(const char* text, int64_t len, int64_t n, int64_t* ids, double* xyz);
int dgb_msh4_elements(const char* text, int64_t len, int64_t n, int32_t* type, int32_t* entity_dim,
                      int32_t* entity_tag, int64_t* offsets, int64_t* nodes, int64_t cap);
/* Optional sum-factorised path for a mesh of one hexahedron block (hexahedron bases are
 * tensor products of the 1-D Lagrange basis on the nodes 0, 1, interior: hybrid/elements.py:
 * 199-274, 325-456).  line_tables: 173 doubles, in order bq[5][4], dq[5][4] (1-D basis and
 * derivative at the volume Gauss points), bqT[4][5], dqT[4][5] (transposes), bf[4][4], df[4][4]
 * (at the face Gauss points), bfT[4][4], d0[4], d1[4] (derivatives at 0 and 1), m1i[4][4] (the
 * inverse of the 1-D mass matrix), w1[5] (1-D volume Gauss weights on [0, 1]), p1d[4][4] (the
 * nodal projector onto span{1, xi}, whose threefold tensor product is the sensor's P1
 * projector), each block using its leading (points x nodes) entries; lex2node: 64 ints mapping lexicographic
 * (x fastest) node positions to element node indices; perm: [codes][face_points] map from the
 * owner's face-point order to the side element's canonical face grid. */
int dgb_plan_set_hex(dgb_plan* plan, const double* line_tables, const int32_t* lex2node, int num_codes,
                     int face_points, const uint8_t* perm);

/* Optional, after dgb_plan_set_hex: elements whose map is affine (a parallelepiped; the
 * inverse Jacobian is the same at every volume point).  For them the kernels use the constant
 * inverse Jacobian jinv[E][9] and det J det[E] instead of the per-point metrics, and apply
 * M^-1 = coef * (m1i (x) m1i (x) m1i) with coef[E] = sliver scale / det J by three 1-D passes
 * instead of reading the element's dense M^-1 (hybrid/geometry.py:181-192 computes the same
 * matrix by quadrature).  affine[E] is 1 for those elements, 0 for the others. */
int dgb_plan_set_hex_affine(dgb_plan* plan, const uint8_t* affine, const double* coef, const double* jinv,
                            const double* det);
/* Affine elements of a block on the dense (any element type) path: where affine[e] is 1 the
 * kernels use the constant inverse Jacobian jinv[e][9], w_q |det J| = ref_weights[q] * det[e]
 * and M^-1 = coef[e] * ref_inv_mass (coef = sliver scale / |det J|, ref_inv_mass the inverse of
 * B^T diag(ref_weights) B, [Np][Np]) instead of the per-element tables; equal to them to
 * round-off (hybrid/geometry.py:139-203 builds the per-element ones).  Not for the
 * sum-factorised hexahedron path (dgb_plan_set_hex_affine). */
int dgb_plan_set_block_affine(dgb_plan* plan, int block, const uint8_t* affine, const double* coef,
                              const double* jinv, const double* det, const double* ref_weights,
                              const double* ref_inv_mass);
/* Ensembles of independent cases in one plan (the mesh is the disjoint union of the cases'
 * meshes; no face joins two cases).  cases is [num_cases][3 + nvars]: dynamic viscosity,
 * thermal conductivity, wall temperature (used where the plan's parameters ask for an
 * isothermal wall) and the far-field primitive state; element_case[b] gives the case of each
 * element of block b.  These replace the plan-wide values of dgb_params in the viscous flux,
 * the boundary ghosts and the stable time step; everything else (gamma, gas constant, BR2
 * penalty, boundary tags, limiter settings) stays shared.  One dt serves all cases. */
int dgb_plan_set_cases(dgb_plan* plan, int num_cases, const double* cases, const int32_t* const* element_case);
int dgb_plan_finalize(dgb_plan* plan);
int dgb_plan_destroy(dgb_plan* plan);
/* Replace the physics/boundary/limiter constants of a finalized plan (same mesh and degree);
 * the reference passes boundary_state per call (hybrid/spatial.py:236). */
int dgb_plan_update_params(dgb_plan* plan, const dgb_params* params);

/* HybridEulerOperator.rhs (hybrid/spatial.py:236-249) -> inviscid_out;
 * HybridNavierStokesOperator.viscous_rhs (hybrid/navier_stokes.py:326-336) -> viscous_out.
 * Either output may be NULL (not computed / not written). */
int dgb_rhs(dgb_plan* plan, const dgb_state* U, const dgb_state* inviscid_out,
            const dgb_state* viscous_out, void* stream);
/* Physical coordinates of every face point, [F][nq][3] for one face type (the moment arms of
 * dgb_wall_forces). */
int dgb_plan_set_face_points(dgb_plan* plan, int face_type, const double* points);
/* Surface forces on the boundary faces whose tag is in wall_tags (hybrid/aerodynamics.py:149-250):
 * evaluates the right-hand side of U (for the face traces, gradients and BR2 lifts; boundary
 * descriptor as set by dgb_plan_update_params) and writes to the DEVICE array out[12]: pressure
 * force sum p n dA (3), its moment about moment_center (3), viscous force -sum (tau . n) dA
 * (3) and its moment (3); n is the face normal out of the fluid.  Deterministic (fixed-order
 * reductions). */
int dgb_wall_forces(dgb_plan* plan, const dgb_state* U, const int32_t* wall_tags, int n_wall_tags,
                    const double* moment_center, double* out, void* stream);
/* Autotuner of the dense (any element type) kernels: times the trace, volume and finalize
 * launches on state U for each block's threads-per-element width in {16, 32, 64, 128} (best of
 * `reps` runs, one coordinate sweep) and keeps the fastest in the plan.  widths (optional,
 * [3][DGB_MAX_BLOCKS]) receives the choice per kernel (trace, volume, finalize) and block; all
 * zeros on the sum-factorised hexahedron path, whose launches are fixed.  Synchronises the
 * stream. */
int dgb_plan_autotune(dgb_plan* plan, const dgb_state* U, int reps, int* widths, void* stream);
/* Execution form of the sum-factorised hexahedron right-hand side (no reference counterpart; the
 * results agree to round-off): enable = 1 (the default) runs it as three launches, the traces,
 * one face kernel (HLLC, BR2 jumps, both sides' local lifts and the viscous face flux) and one
 * element kernel (nodal lift, volume terms, face terms, M^-1 and the stage update, with the lift
 * and the residuals kept on chip); enable = 0 runs the six-launch form (traces, face flux, lift,
 * volume, viscous face flux, finalize). */
int dgb_plan_set_fused(dgb_plan* plan, int enable);
/* Inviscid volume integrals of the dense blocks on the tensor cores (replaces the einsum
 * contractions of HybridEulerOperator._volume_terms, hybrid/spatial.py:47-72, for those blocks):
 * a tcgen05 kernel with three-term TF32 products (about float32 accuracy) and bulk-copied
 * element tiles.  It applies to plans in precision mode 1 (mixed) without viscous terms, to
 * blocks with an even node count of at most 40 and at most 128 volume points, 5 variables
 * (prisms and tetrahedra up to P3); other blocks keep the CUDA-core kernel.  enable = 0 turns it
 * off.  blocks_out (optional) receives how many blocks use it.  Packs the block's constant
 * operands on the device the first time (synchronises the device). */
int dgb_plan_set_tensor_cores(dgb_plan* plan, int enable, int* blocks_out);
/* Error bits that kernels with bounded waits record on the device (1: a wait on the tensor
 * cores or the bulk-copy engine ran out of time; the kernel released its tensor memory and
 * returned without writing that tile).  Copies the word to host *out; reset = 1 clears it.
 * Synchronises the device. */
int dgb_plan_device_errors(dgb_plan* plan, int* out, int reset);

/* HybridSSPRK3.stable_dt (hybrid/time_integration.py:93-169): writes the clipped dt
 * to the device double *dt_out. */
int dgb_stable_dt(dgb_plan* plan, const dgb_state* U, double cfl, double* dt_out, void* stream);

/* HybridPositivityLimiter.__call__ (hybrid/limiter.py:100-147), in place. */
int dgb_positivity(dgb_plan* plan, const dgb_state* U, void* stream);

/* HybridTroubledCellSensor.__call__ (hybrid/limiter.py:165-185): sensor values [E_b] per block
 * (device doubles, may be NULL) and HybridMOODSubcellLimiter.troubled (hybrid/limiter.py:285-300)
 * flags [E_b] per block (device uint8, may be NULL). */
int dgb_troubled(dgb_plan* plan, const dgb_state* U, double* const* sensor_out,
                 uint8_t* const* flags_out, void* stream);

/* HybridSSPRK3.state_admissibility (hybrid/time_integration.py:291-312) into *status (device). */
int dgb_admissibility(dgb_plan* plan, const dgb_state* U, dgb_status* status, void* stream);

/* HybridSSPRK3.checked_step (hybrid/time_integration.py:441-583), in place on U.
 * limiter 0/1: three SSP-RK3 stages, each RHS -> blend -> positivity -> admissibility;
 *   *status (device) receives valid1&valid2&valid3 and the minima over the stages.
 * limiter 2 (MOOD, needs dgb_plan_enable_mood): each stage RHS (inviscid and viscous) ->
 *   Euler candidate and unlimited blend -> troubled flags on the unlimited state -> subcell
 *   recompute -> positivity -> blend -> positivity -> admissibility; *status receives the
 *   last stage's admissibility, as the reference's MOOD branch returns. */
int dgb_ssprk3_step(dgb_plan* plan, const dgb_state* U, double dt, dgb_status* status, void* stream);

/* dgb_ssprk3_step as one CUDA graph: the first call (and any call whose state pointers, dt or
 * status pointer differ from the previous one, or that follows a change of the plan's
 * parameters, MOOD set-up or predictor) captures the step's kernels on a private stream and
 * instantiates them; every call then launches the graph on `stream`.  Same results as
 * dgb_ssprk3_step (the same kernels in the same order).  A replay is one launch instead of the
 * step's several hundred, which matters when the step is short; keep dt and the state buffers
 * fixed across steps to replay without capturing again. */
int dgb_ssprk3_step_graph(dgb_plan* plan, const dgb_state* U, double dt, dgb_status* status, void* stream);

/* MOOD subcell finite-volume tables of one element block (hybrid/subcell.py:216-396):
 * 64 subcells, NI internal and NB boundary subfaces of the reference subdivision. */
typedef struct {
  int num_subcells, num_internal, num_boundary;
  const double* projection;       /* [E][S][Np] metric-weighted DG -> subcell means      */
  const double* reconstruction;   /* [E][Np][S] volume-weighted least-squares inverse    */
  const double* volumes;          /* [E][S]                                              */
  const double* centers;          /* [E][S][3]                                           */
  const double* internal_normals; /* [E][NI][3] owner -> neighbour                       */
  const double* internal_areas;   /* [E][NI]                                             */
  const double* boundary_normals; /* [E][NB][3] outward                                  */
  const double* boundary_areas;   /* [E][NB]                                             */
  const int32_t* internal_owner;  /* [NI] */
  const int32_t* internal_neighbor; /* [NI] */
  const int32_t* csr_ptr;         /* [S+1] internal subfaces of each subcell             */
  const int32_t* csr_face;        /* [2 NI]                                              */
  const double* boundary_basis;   /* [NB][Np] DG basis at the boundary subface centres   */
  const int32_t* gather;          /* [NB] subcell read for a boundary subface            */
  const int32_t* scatter;         /* [NB] subcell updated by a boundary subface, -1 none */
} dgb_subcell_block_desc;

/* MOOD tables; may be given before or after dgb_plan_finalize.  osub/nsub: [F][16] boundary
 * subfaces of the owner and of the neighbour (matched to the owner's), -1 on boundary faces. */
int dgb_plan_set_subcells(dgb_plan* plan, int block, const dgb_subcell_block_desc* desc);
int dgb_plan_set_subcell_faces(dgb_plan* plan, int face_type, const int32_t* osub, const int32_t* nsub);
int dgb_plan_enable_mood(dgb_plan* plan);

/* The same MOOD tables built on the device (HybridSubcellFV.__init__, hybrid/subcell.py:277-396),
 * in place of dgb_plan_set_subcells / dgb_plan_set_subcell_faces.  The reference subdivision of
 * the block's element type is described once, host pointers:
 *   - the subcells' P2 volume rule (Qs points per subcell, each weight times the subcell's
 *     affine reference-volume factor), the DG basis and the geometry-basis gradients at the
 *     mapped points, the geometry basis at the subcell vertices;
 *   - the subcell vertex lists and the internal and boundary subfaces (3 or 4 vertices, -1 past
 *     a triangle's third), with the index tables of dgb_subcell_block_desc.
 * geometry_nodes: host [E][num_geometry_nodes][3], the block's geometry-map nodes.  Per element
 * the device forms |det J| at the mapped points, the subcell volumes and centres, the
 * metric-weighted projection, its volume-weighted least-squares left inverse (Gram matrix
 * inverted by Gauss-Jordan) and the subface normals, areas and centres, one CTA per element.
 * A Gram matrix that is not positive definite fails with DGB_ERR_ARGUMENT. */
typedef struct {
  int num_subcells;               /* S = 64 */
  int num_points;                 /* Qs */
  int num_geometry_nodes;         /* ng of the geometry map */
  int num_vertices;               /* V, subcell vertices */
  int cell_size;                  /* vertices per subcell: 8, 6 or 4 */
  int num_internal, num_boundary; /* NI, NB */
  const double* rule_weights;     /* [S][Qs] */
  const double* point_basis;      /* [S][Qs][Np] */
  const double* point_geometry_grad; /* [S][Qs][ng][3] */
  const double* vertex_geometry;  /* [V][ng] */
  const int32_t* cells;           /* [S][cell_size] */
  const int32_t* internal_faces;  /* [NI][4] */
  const int32_t* boundary_faces;  /* [NB][4] */
  const int32_t* internal_owner;  /* [NI] */
  const int32_t* internal_neighbor; /* [NI] */
  const int32_t* boundary_owner;  /* [NB] */
  const int32_t* csr_ptr;         /* [S+1] */
  const int32_t* csr_face;        /* [2 NI] */
  const double* boundary_basis;   /* [NB][Np] */
  const int32_t* gather;          /* [NB] */
  const int32_t* scatter;         /* [NB] */
} dgb_subcell_reference;

int dgb_plan_build_subcells(dgb_plan* plan, int block, const dgb_subcell_reference* ref,
                            const double* geometry_nodes);
/* Neighbour subfaces matched to the owner's by physical centre on the device (subcell.py:
 * 473-533): osub [F][16] the owner's boundary subfaces, ncand [F][16] the neighbour's boundary
 * subfaces on its parent face in reference order (-1 on boundary faces), host.  Centres are
 * taken relative to each side's face centre, so periodic partners match; a face whose 16
 * nearest partners are not distinct or lie farther than 2e-6 of the face's scale fails with
 * DGB_ERR_ARGUMENT.  Needs dgb_plan_build_subcells on the blocks of both sides first. */
int dgb_plan_match_subcell_faces(dgb_plan* plan, int face_type, const int32_t* osub, const int32_t* ncand);

/* HybridSubcellFV.recompute (hybrid/subcell.py:855-950): base state, Euler DG candidate,
 * dt, optional additional rhs (viscous, projected onto the subcells) and troubled flags
 * [E_b] per block (device uint8) -> out (device state).  No positivity limiting. */
int dgb_subcell_recompute(dgb_plan* plan, const dgb_state* base, const dgb_state* candidate, double dt,
                          const dgb_state* additional_rhs, uint8_t* const* troubled, const dgb_state* out,
                          void* stream);

/* Tracing (no reference counterpart; the reference only prints wall-clock progress,
 * run_hybrid_sphere.py:366-390): runs one dgb_rhs with CUDA events around each kernel
 * stage and writes the stage durations in milliseconds to host ms_out[DGB_RHS_STAGES]
 * (traces, face flux, BR2 lift, volume, viscous face flux, finalize; on the dense path the
 * lift is part of the volume stage and its entry is 0).  Synchronises the stream. */
enum { DGB_RHS_STAGES = 6 };
int dgb_rhs_profile(dgb_plan* plan, const dgb_state* U, float* ms_out, void* stream);
/* The same for the right-hand side as an SSP-RK stage forms it (the stage update fused into
 * the last kernel, with dt = 0 into plan scratch), split = 1 with the viscous residual kept
 * apart as the MOOD step of the six-launch form needs it, split = 0 as one residual (the
 * MOOD step of the fused form, and every step without MOOD). */
int dgb_rhs_profile_stage(dgb_plan* plan, const dgb_state* U, int split, float* ms_out, void* stream);

/* Allocation-free CFL time step for one element block.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory when they ask for a time step: host
 * codes or coupling frameworks that hand the library a fixed device-memory pool and
 * forbid allocations behind their back, and time loops that must not call cudaMalloc
 * (an allocation synchronises the device and can fail once the pool is reserved).
 * It needs no plan: U is the block's device state (E, Np, nvars) float64, length the
 * device array of per-element characteristic lengths (hybrid/time_integration.py:49-91),
 * dt_out a device double; the result is the same clipped dt as dgb_stable_dt
 * (hybrid/time_integration.py:93-169).  For a mesh of several blocks, call it per block
 * and take the smallest dt.
 *
 * Scratch: a file-scope device array of 2^20 doubles (8 MiB) that every GPU which loads
 * the library keeps until the process exits; at most 1048576 elements per call (larger
 * blocks are rejected with DGB_ERR_ARGUMENT, and so is a negative degree).  The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress) with the device
 * current; make that first call before any stream capture.  Under CUDA's default lazy
 * module loading that first call is also when the driver loads this code's module on the
 * device and with it the 8 MiB array: that one time the driver itself takes device
 * memory.  A caller that reserves its whole pool up front should make the first call
 * before reserving it (or run with CUDA_MODULE_LOADING=EAGER, which loads the module, and
 * the array, when the library is loaded).  All calls share the array: calls whose kernels
 * overlap on the GPU (different streams or threads) race on it.  Errors are reported by
 * dgb_noalloc_last_error(). */
int dgb_stable_dt_noalloc(const double* U, const double* length, int num_elements, int num_nodes, int nvars,
                          int degree, double gamma, double gas_constant, double dynamic_viscosity,
                          double thermal_conductivity, double br2_penalty, double cfl, double* dt_out,
                          void* stream);
const char* dgb_noalloc_last_error(void);

/* ---- Finite-rate chemistry (operator-split source), hybrid/chemistry/ ----------------
 *
 * A reaction mechanism as dense tables, filled from the mechanism's species and
 * reactions (ReactionMechanism.__init__, hybrid/chemistry/mechanism.py:58-123; the
 * Air-11 Park data of hybrid/chemistry/air11_park.py:20-311).  Host pointers; the
 * library copies them.  Species count: 3 or 11 (the kernels are compiled for those);
 * at most DGB_CHEM_MAX_REACTIONS reactions, each with at most 3 distinct reactant,
 * 3 distinct product and 6 distinct net-stoichiometry species. */
enum { DGB_CHEM_MAX_SPECIES = 11, DGB_CHEM_MAX_REACTIONS = 32 };
typedef struct {
  int num_species, num_reactions;
  const double* molar_mass;        /* [ns] kg/mol */
  const double* nu_forward;        /* [nr][ns] reactant stoichiometry nu' */
  const double* nu_reverse;        /* [nr][ns] product stoichiometry nu'' */
  const double* efficiency;        /* [nr][ns] third-body efficiencies alpha_M */
  const double* arrhenius;         /* [nr][3] A, b, theta of kf = A T^b exp(-theta/T) (SI) */
  const int* third_body;           /* [nr] 0/1 */
  const int* forward_mode;         /* [nr] controlling temperature: 0 T, 1 sqrt(T Tv), 2 Tv */
  const int* reverse_mode;         /* [nr] */
  const double* nasa_range;        /* [ns][3] t_low, t_mid, t_high */
  const double* nasa_coeffs;       /* [ns][2][7] low-range then high-range a0..a6 */
} dgb_chem_mechanism;

/* ReactingFlowCoupler.__init__ (hybrid/chemistry/coupling.py:26-71) without relaxation
 * (single temperature, relaxation=None). */
typedef struct {
  int max_newton_iters;            /* default 12 */
  int dimensionless;               /* 0/1 */
  double reference_temperature;    /* K, default 300 */
  double reference_pressure;       /* Pa, default 101325 */
  double reference_length;         /* m, default 1 */
  double gamma;                    /* default 1.4 */
} dgb_chem_params;

typedef struct dgb_chem dgb_chem;

int dgb_chem_create(const dgb_chem_mechanism* mechanism, const dgb_chem_params* params, dgb_chem** out);
int dgb_chem_destroy(dgb_chem* chem);

/* ReactingFlowCoupler.react_block (hybrid/chemistry/coupling.py:179-197, per node
 * _react_single_cell :116-177 with PointImplicitIntegrator.step,
 * hybrid/chemistry/integrator.py:31-104): U and out are device arrays
 * (num_elements, num_nodes, nvars) float64 with the species partial densities in
 * columns 5 .. 5+ns-1; out may equal U.  Columns 0..4 are copied unchanged.  dt is the
 * time step (dimensionless when the coupler is); dt_per_element, when not null, is a
 * device array of num_elements steps that replaces dt (local time stepping).
 * nvars < 5 + ns is DGB_ERR_ARGUMENT (the reference raises ValueError). */
int dgb_react_block(dgb_chem* chem, const double* U, double* out, int64_t num_elements, int num_nodes,
                    int nvars, double dt, const double* dt_per_element, void* stream);

/* ---- Learned troubled-cell predictor (no reference counterpart) -----------------------
 *
 * A small MLP (8 features -> 64 -> 64 -> 64 -> 1, ReLU, sigmoid) that predicts from a stage's
 * base state which elements the MOOD a-posteriori test (hybrid/limiter.py:285-300) will flag,
 * so that they go to the subcell scheme without the failed high-order attempt.  The test
 * stays the fallback and the arbiter.  Parameters are DGB_MLP_PARAMS floats in the order
 * W1[8][64], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4; norm is the
 * features' mean[8] then 1/std[8].  All arrays are device arrays. */
enum { DGB_MLP_FEATURES = 8, DGB_MLP_PARAMS = 8961 };

/* Features of every element of U, (sum of E, 8) float32 in block order. */
int dgb_mlp_features(dgb_plan* plan, const dgb_state* U, float* features, void* stream);
/* Inference with float16 weights and float32 accumulation: prob[n] and/or flag[n] = prob > threshold. */
int dgb_mlp_infer(const void* weights_f16, const float* norm, const float* features, int64_t n, float threshold,
                  float* prob, uint8_t* flag, void* stream);
/* One Adam step (step >= 1) on the float32 weights over the samples features[index[0..batch)],
 * labels 0/1, binary cross-entropy with positive samples weighted by pos_weight.  grad
 * (DGB_MLP_PARAMS, zero on entry) is cleared again; weights_f16 (optional) receives the updated
 * weights; loss (optional, device float) accumulates the batch loss. */
int dgb_mlp_train_step(float* weights, float* grad, float* adam_m, float* adam_v, void* weights_f16,
                       const float* norm, const float* features, const uint8_t* labels, const int* index,
                       int batch, float pos_weight, float lr, int step, float* loss, void* stream);
/* Use the predictor inside dgb_ssprk3_step's MOOD stages: mode 0 off, 1 learned (predicted
 * elements skip the a-posteriori test and go to the subcell scheme; on the fused hexahedron
 * path they also skip their high-order update), 2 evaluate (every element
 * is tested and the step is the plain one; the prediction is only counted).  The weight and
 * norm arrays must outlive their use. */
int dgb_plan_set_predictor(dgb_plan* plan, const void* weights_f16, const float* norm, float threshold, int mode);
/* Host int64[5]: [0] unused (0), [1] predicted, [2] missed (tested troubled but not predicted),
 * [3] false positives and [4] hits (both counted in mode 2 only); reset clears them. */
int dgb_plan_predictor_counts(dgb_plan* plan, int64_t* counts, int reset);

/* ReactionMechanism.net_production_rates (hybrid/chemistry/mechanism.py:159-220) at
 * count independent samples, single temperature: rho (count, ns) and T (count) device
 * arrays; omega (molar rates), wdot (mass rates after the mass-conserving correction) and
 * jacobian (count, ns, ns) = d wdot / d rho are device outputs, each may be null. */
int dgb_chem_rates(dgb_chem* chem, const double* rho, const double* T, int64_t count, double* omega,
                   double* wdot, double* jacobian, void* stream);

/* ---------------------------------------------------------------- midplane rasteriser
 * (hybrid/gui/gpu_rasterizer.py:18-344) into a headless RGBA buffer.  The host locates each
 * pixel on the cut plane: pixel_block[p] (-1 outside the mesh), pixel_element[p] and the
 * solution-basis weights pixel_weights[p][max_nodes] (float32) of that element at the pixel.
 * Device arrays throughout. */
typedef struct {
  int nx, ny, max_nodes;
  int block_nodes[DGB_MAX_BLOCKS];   /* nodes per element of each block */
  const int32_t* pixel_block;
  const int32_t* pixel_element;
  const float* pixel_weights;
  const uint8_t* body_mask;          /* 1: paint the background colour (the body) */
  const uint8_t* grad_mask;          /* 1: no schlieren gradient (next to the body) */
  const uint8_t* luts;               /* [2][256][4]: the field palette, the temperature palette */
  uint8_t background[4];
  double dx, dy;                     /* pixel spacing */
} dgb_raster_desc;

/* Renders mode 0 schlieren, 1 density, 2 pressure, 3 Mach, 4 temperature of U into rgba
 * [ny][nx][4] (row 0 at the top); grid is scratch [ny][nx][5] float64 (rho, u, v, w, p). */
int dgb_raster_render(const dgb_raster_desc* desc, const dgb_state* U, int nvars, double gamma, int mode,
                      double vmin, double vmax, double* grid, uint8_t* rgba, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DGB200_H */
