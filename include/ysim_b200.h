/* ysim_b200.h -- C ABI of the B200 (sm_100a) implementation of ysim's
 * per-substep cloth hot path.
 *
 * This is the drop-in boundary for the reference's empty `CUDA` backend slot
 * (include/sim/core_types.hpp:9).  Plain pointers and sizes only; no CUDA or
 * torch types appear in a signature (streams are passed as void*).  Every call
 * returns ys_status (0 = ok, negative = error, see ys_last_error()).  Device
 * conditions (overflow, non-finite output, iteration caps) are latched in a
 * per-scene flag word read with ys_scene_stats().
 *
 * Threading: one scene = one CUDA stream; a scene is not thread-safe, distinct
 * scenes may be driven from distinct threads.
 */
#ifndef YSIM_B200_H
#define YSIM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int ys_status;
#define YS_OK 0
#define YS_ERR_BAD_ARG (-1)
#define YS_ERR_CUDA (-2)
#define YS_ERR_STATE (-3)
#define YS_ERR_CAPACITY (-4)

/* Device flag bits (ys_scene_stats out[5]); the reference's QueryFlag
 * (bvh.hpp:396-400) and anomalyFlag (symplectic_system.hpp:184) folded into
 * one word. */
#define YS_FLAG_NONFINITE 1u
#define YS_FLAG_STACK_OVF 2u
#define YS_FLAG_PAIR_OVF 4u
#define YS_FLAG_ITER_CAP 8u
#define YS_FLAG_CONTACT_OVF 16u

/* BehaviorType values (mesh_state.hpp:108-124). */
#define YS_TRIANGULAR_CLOTH 0u
#define YS_FAST_GRID_CLOTH 1u
#define YS_RIGID 3u
#define YS_FLOAT 4u
#define YS_KINEMATIC 7u

/* Mesh flags (GeneralMesh::isStatic / collidable / selfCollide, scene.hpp:58). */
#define YS_MESH_STATIC 1u
#define YS_MESH_COLLIDABLE 2u
#define YS_MESH_SELF_COLLIDE 4u

/* ColliderKind (include/sim/collision_pod.hpp; YSIM_COLLIDER_*,
 * src/metal/common_types.metalh:80-84). */
#define YS_COLLIDER_MESH 0u
#define YS_COLLIDER_SPHERE 1u
#define YS_COLLIDER_BOX 2u
#define YS_COLLIDER_CYLINDER 3u
#define YS_COLLIDER_PLANE 4u

/* AnalyticShape (include/sim/collision_pod.hpp:295-309; mirror in
 * src/metal/common_types.metalh:42-52), 96 bytes: world centre and radius
 * (sphere radius, cylinder radius), half extents (box half extents, ellipsoid
 * semi-axes) and cylinder half height, orientation (w, x, y, z) local to
 * world, centre and orientation at the start of the step, collider kind,
 * owning mesh index, behaviour, flags (bit 0: collidable).  Local frame: a
 * plane is the half-space y <= 0, a cylinder's axis is +y. */
typedef struct ys_analytic_shape {
    float center_radius[4];
    float half_ext_height[4];
    float rot_quat[4];
    float prev_center[4];
    float prev_rot_quat[4];
    uint32_t kind, obj_index, behavior, flags;
} ys_analytic_shape;

/* Self-collision row source: off, the reference default CPU-spatial-hash
 * semantics (Simulator::useCpuShSelf, simulator.hpp:93; CpuSpatialHash
 * spatial_hash.hpp:1946-1989) or BVH self queries (checkSelfCollisions,
 * bvh.hpp:1842-1848). */
#define YS_SELF_OFF 0u
#define YS_SELF_HASH 1u
#define YS_SELF_BVH 2u

/* Morton normalisation of the scene's trees.  REFERENCE scales each axis by
 * the mesh box's own width (fillMortons_Tri, src/metal/bvh.metal:42-63), which
 * reproduces the reference's tree node for node.  CUBE (the default) scales
 * all axes by the largest width: on a flat, jittered sheet the per-axis form
 * spreads the thin axis's jitter over all ten of its bits, so the tree splits
 * on it at every third level into siblings covering the same area, and each
 * query descends both.  The candidate sets, contacts and positions are the
 * same under both layouts (every leaf box is the same; only the order of the
 * descent changes). */
#define YS_TREE_REFERENCE 0
#define YS_TREE_CUBE 1

/* Tree builder.  KARRAS: buildTree_Tri (src/metal/bvh.metal:352-393), then
 * the boxes bottom-up (the reference default).  APETREI: agglomerativeBuild_Tri
 * + agglomerativeSwapRoot (bvh.metal:884-1199; BVH::useAgglomerative,
 * bvh.hpp:292-295): topology and boxes in one pass, one thread per leaf
 * climbing to the root, the root moved to slot 0.  Its tree is the
 * reference's Apetrei tree node for node; runs of equal Morton codes split by
 * primitive index, so every node has one parent. */
#define YS_BUILD_KARRAS 0
#define YS_BUILD_APETREI 1

/* Simulator / SymplecticSystem parameters: subh, kair, kd
 * (symplectic_system.hpp:191-198), gravity (Scene::environment), margin and
 * radius (simulator.hpp:180-181), substeps per frame, BVH rebuild period in
 * frames (simulator.hpp:3253), self-collision mode, collision budget per
 * vertex (approxColsPerPoints, scene.hpp:1139). */
typedef struct ys_sim_params {
    float subh, kair, kd;
    float gravity[3];
    float margin, radius;
    uint32_t substeps, rebuild_frames, self_mode, cols_per_point;
} ys_sim_params;

/* One mesh (GeneralMesh: MeshState + MeshAdjacency + behavior params,
 * scene.hpp / mesh_state.hpp / collision_pod.hpp:349-396).  Arrays are host
 * pointers in the reference layout: x, v = 3 floats per vertex; facets = 3
 * local vertex ids per triangle; mass, mask = one float per vertex.
 * k* / thickness: ClothBehaviorParams (stretch, shear, bend, thickness) or
 * FastGridClothBehaviorParams (kstretch, kshear, kbend, thickness) with
 * grid_n = particleNum1D and grid_rest = stretchRestX/Y, shearRestA/B,
 * bendRestX/Y.  group: meshes only collide with meshes of the same group
 * (independent scene instances in one batched scene). */
typedef struct ys_mesh_desc {
    uint32_t behavior, flags, num_vertices, num_facets;
    const float* x;
    const float* v;
    const float* mass;
    const float* mask;
    const uint32_t* facets;
    float kstretch, kshear, kbend, thickness;
    uint32_t grid_n;
    float grid_rest[6];
    uint32_t group;
} ys_mesh_desc;

typedef struct ys_scene ys_scene;
typedef struct ys_lbvh ys_lbvh;
typedef struct ys_shash ys_shash;
typedef struct ys_adjoint ys_adjoint;

/* Last error message of the calling thread. */
const char* ys_last_error(void);
/* Library version string. */
const char* ys_version(void);

/* ---- Scene (Scene<CUDA,PR>::pack, scene.hpp:783-1180) ---------------- */
ys_status ys_scene_create(ys_scene** out, const ys_sim_params* params, int device);
ys_status ys_scene_destroy(ys_scene* s);
ys_status ys_scene_add_mesh(ys_scene* s, const ys_mesh_desc* mesh, int* index_out);
/* Upload, build adjacency (MeshAdjacencyInitializer, mesh_state.hpp:236-411),
 * build every tree (BroadPhase::build, bvh.hpp:2537-2590). */
ys_status ys_scene_pack(ys_scene* s);

/* ---- Reference stage surfaces (one call per Simulator::update stage) --- */
/* Frame preamble: periodic rebuild (simulator.hpp:3253-3261) + environment
 * forces (applyEnvironmentForces, simulator.hpp:3123-3166); no-op mid-frame. */
ys_status ys_frame_preamble(ys_scene* s);
/* BroadPhase::refitSwept (bvh.hpp:2752-2806): swept leaves + bottom-up. */
ys_status ys_broad_refit(ys_scene* s);
/* BroadPhase::detectCollisions (bvh.hpp:2853-2949) with the hybrid self pass
 * (simulator.hpp:3678-3701): writes broad rows. */
ys_status ys_broad_detect(ys_scene* s);
/* BruteForce::narrowAndSortByVertices (bruteforce.hpp:311-383). */
ys_status ys_narrow_and_sort(ys_scene* s);
/* SymplecticSystem::snapshotXPrev (symplectic_system.hpp:230-250). */
ys_status ys_snapshot_xprev(ys_scene* s);
/* SymplecticSystem::update (symplectic_system.hpp:341-409). */
ys_status ys_system_update(ys_scene* s);

/* ---- Whole substeps ---------------------------------------------------- */
/* n substeps through the staged kernels above (one launch group per stage). */
ys_status ys_scene_step_staged(ys_scene* s, uint32_t n);
/* n substeps through the fused path: refit + one kernel doing detect,
 * narrow, per-vertex contacts, spring forces and integration (same results
 * as the staged path). */
ys_status ys_scene_step(ys_scene* s, uint32_t n);
/* Record the fused path's per-vertex contacts for inspection (slower). */
ys_status ys_scene_set_record(ys_scene* s, int record);
/* Replay each fused substep as a captured CUDA graph (default on; substeps
 * that rebuild trees, record contacts or time kernels run eagerly). */
ys_status ys_scene_set_graphs(ys_scene* s, int on);
/* Register cap of the fused substep kernel, as CTAs per SM (8: 64 registers,
 * 7: 72, 4: uncapped).  The results are the same for every value; the speed
 * depends on the scene (the self-colliding 262k-vertex cloth runs fastest at 7,
 * the batched FastGrid instances at 8).  No counterpart in the reference (its Metal pipelines have
 * fixed threadgroup sizes). */
ys_status ys_scene_set_fused_variant(ys_scene* s, int min_blocks);
/* Thread order of the fused substep kernel, for every size class.  Its
 * threads take the working vertices (cloth, moving or querying; static
 * obstacles are left out), mesh after mesh:
 *   YS_ORDER_MORTON (default): in Morton order within each mesh, recomputed
 *     from the positions at every tree rebuild, so a warp's 32 vertices are a
 *     compact patch whose descents and candidate faces overlap;
 *   YS_ORDER_VERTEX: thread i takes vertex i;
 *   YS_ORDER_TILE: each CTA takes one 16 x 8 tile of a FastGridCloth (other
 *     meshes in vertex order, each from a CTA boundary); the tile's positions
 *     and velocities with a 2-vertex halo come into shared memory by TMA, and
 *     each stencil spring with an end in the tile is evaluated once for both
 *     of its ends (890 spring evaluations per tile instead of 1536).
 * The results are the same, bit for bit, in every order.  No counterpart in
 * the reference (one Metal thread per vertex id). */
#define YS_ORDER_VERTEX 0
#define YS_ORDER_MORTON 1
#define YS_ORDER_TILE 2
ys_status ys_scene_set_thread_order(ys_scene* s, int order);
/* Autotuner: times each variant on the scene's current state (reps launches
 * each; the kernel only writes the next-state buffers and the running totals
 * are restored, so the scene does not advance), keeps the fastest, and
 * reports it (*chosen) and the mean milliseconds per variant (ms_out[3], in
 * the order 8, 7, 4; may be null).  No counterpart in the reference. */
ys_status ys_scene_autotune(ys_scene* s, uint32_t reps, int* chosen, float* ms_out);
/* The fused substep runs one launch per size class of the working meshes
 * (cloth, moving or querying meshes with at most 4096, 16384, 65536 vertices,
 * and larger; a batch of instances of mixed sizes spans several).  Each
 * class has its own register-cap variant and thread order. */
typedef struct ys_fused_class {
    uint32_t max_mesh_vertices;  /* the class's bound on a mesh's vertex count */
    uint32_t meshes, vertices;   /* working meshes and vertices in the class */
    int32_t ctas_per_sm;         /* chosen variant (8, 7 or 4) */
    int32_t thread_order;        /* chosen thread order: YS_ORDER_VERTEX, _MORTON or _TILE */
    float ms[3][3];              /* mean ms per launch: [vertex, Morton, tile order][8, 7, 4] */
} ys_fused_class;
/* Per-class autotuner: times every variant under each thread order on each
 * class's launch over the current state (the scene does not advance), keeps
 * the fastest pair per class and reports the classes (out: up to cap
 * records; *nclasses: the number of classes, 4).  No counterpart in the
 * reference. */
ys_status ys_scene_autotune_classes(ys_scene* s, uint32_t reps, ys_fused_class* out, uint32_t cap,
                                    uint32_t* nclasses);
/* Analytic collider (GeneralMesh::colliderKind and transform): kind
 * YS_COLLIDER_SPHERE / BOX / CYLINDER / PLANE (YS_COLLIDER_MESH: triangles,
 * the default), centre, local half extents (sphere: semi-axes; box: half
 * extents; cylinder: radius max(h[0], h[2]), half height h[1]; plane: unused,
 * may be NULL) and orientation (w, x, y, z).  Before ys_scene_pack it makes
 * the mesh an analytic collider: its triangles are neither queried nor refit,
 * and the vertices of each cloth whose root box meets the collider's box at
 * this substep's detect or the one before are tested against the shape
 * (BroadPhase::detectCollisions markers, bvh.hpp:2886-2941;
 * PackedCollisionData::endAnalyticPairs, scene.hpp:485-530;
 * BruteForce::narrowAnalytic, bruteforce.hpp:245-309), contacts keyed
 * (collider mesh, 0).  After pack it moves the collider: the pose is read at
 * the next frame start, where the previous pose becomes the start of the
 * swept test (Scene::refreshAnalyticShapes, scene.hpp:659-745).  The kind
 * cannot change after pack.  A cloth may be an analytic collider too (the
 * reference's default for a cloth sphere, cube or cylinder primitive): it
 * then descends no tree, is tested against other analytic colliders, keeps
 * its CPU-hash self rows, and is a shape target for other cloths. */
ys_status ys_scene_set_collider(ys_scene* s, int mesh, uint32_t kind, const float center[3], const float half[3],
                                const float rot_wxyz[4]);
/* The scene's analytic shape table as of the last frame start (compact, in
 * mesh order): *num_out entries, min(cap, *num_out) copied to out. */
ys_status ys_scene_colliders(ys_scene* s, ys_analytic_shape* out, uint32_t cap, uint32_t* num_out);
/* Tree layout (YS_TREE_REFERENCE / YS_TREE_CUBE) for every tree the scene
 * builds; call between ys_scene_create and ys_scene_pack.  Replaces the
 * Morton normalisation inside BVH<..>::build (include/sim/bvh.hpp:1194-1301). */
ys_status ys_scene_set_tree_layout(ys_scene* s, int layout);
/* Builder (YS_BUILD_KARRAS / YS_BUILD_APETREI) of every tree the scene builds
 * (BroadPhase::build with Simulator::useAgglomerativeBVH, bvh.hpp:2322-2325);
 * call before ys_scene_pack. */
ys_status ys_scene_set_tree_builder(ys_scene* s, int builder);
ys_status ys_scene_sync(ys_scene* s);
/* CUDA stream of the scene (cudaStream_t) as void*. */
ys_status ys_scene_stream(ys_scene* s, void** stream_out);

/* ---- Inspection --------------------------------------------------------- */
/* which: 0 x, 1 v, 2 xPrev, 3 f (staged path only); packed 3 floats/vertex. */
ys_status ys_scene_get_state(ys_scene* s, int which, float* host_out);
ys_status ys_scene_set_state(ys_scene* s, int which, const float* host_in);
/* out[0] frame, out[1] substep cursor, out[2] broad rows of the last detect,
 * out[3] narrow contacts of the last narrow, out[4] anomaly (0/1),
 * out[5] flag word, out[6] total vertices, out[7] substeps run. */
ys_status ys_scene_stats(ys_scene* s, uint64_t out[8]);
ys_status ys_scene_clear_flags(ys_scene* s);
/* Running totals since pack: out[0] candidate rows, out[1] contacts (fused
 * path). */
ys_status ys_scene_totals(ys_scene* s, uint64_t out[2]);
/* Upload the per-vertex external force buffer (3 floats per vertex) that
 * Simulator::applyEnvironmentForces fills each frame (simulator.hpp:3123-3166).
 * Until the first call (or after a call with NULL) the kernels use g * m. */
ys_status ys_scene_set_external_forces(ys_scene* s, const float* host_ext);
/* Enqueue a device-to-host copy of the current positions (3 floats per
 * vertex) on the scene stream; complete after ys_scene_sync.  host_out
 * should be pinned for an asynchronous copy. */
ys_status ys_scene_read_positions_async(ys_scene* s, float* host_out);
/* CUDA-event timing of the fused path's kernels (refit, fused substep). */
ys_status ys_scene_set_timing(ys_scene* s, int on);
/* out[0] refit ms total, out[1] refit launches, out[2] fused ms total,
 * out[3] fused launches, since ys_scene_set_timing(s, 1). */
ys_status ys_scene_kernel_times(ys_scene* s, double out[4]);
/* Broad rows of the last staged detect (BroadCollision, 32 B each). */
ys_status ys_scene_rows(ys_scene* s, void* host_rows, uint64_t cap, uint64_t* n_out);
/* Per-vertex contacts of the last narrow (staged) or fused step (record on):
 * offsets (num_vertices + 1) and 24-byte records {tobj, tri, nx, ny, nz, d},
 * canonical (tobj, tri) order within each vertex. */
ys_status ys_scene_contacts(ys_scene* s, uint32_t* host_offsets, void* host_contacts, uint64_t cap, uint64_t* n_out);
/* Tree of one mesh: nodes (2N-1, 32 B BVHNode), parents, sorted codes and
 * primitive indices (any pointer may be NULL). */
ys_status ys_scene_tree(ys_scene* s, int mesh, void* nodes, int32_t* parent, uint32_t* codes, uint32_t* idx,
                        uint32_t* num_prims_out);
/* The 4-wide form of a mesh's tree (cube layout) as the last refit left it:
 * *count wide nodes of 128 B (boxes of the four child slots as x, y, z
 * minima then maxima, SoA; child words, >= 0 a wide node, < 0 the
 * complement of a face, 0x7FFFFFFF empty; child count; parent; slot in the
 * parent), the first min(*count, cap) into out.  *count = 0 for the
 * reference layout or a tree never built.  An inspection entry point of this
 * layout; no counterpart in the reference. */
ys_status ys_scene_wide_tree(ys_scene* s, int mesh, void* out, uint32_t cap, uint32_t* count);

/* ---- Differentiable rollouts (adjoint of the substep) --------------------
 * Per-spring parameters of a FastGridCloth (FastGridClothBehaviorParams has
 * three stiffnesses and six rest lengths, collision_pod.hpp:388-396; uniform
 * arrays reproduce it exactly).  Canonical spring order: stretch x
 * (r,c)-(r,c+1), stretch y (r,c)-(r+1,c), shear (r,c)-(r+1,c+1), shear
 * (r,c+1)-(r+1,c), bend x (r,c)-(r,c+2), bend y (r,c)-(r+2,c), each family
 * row-major.  Device pointers. */
ys_status ys_scene_set_grid_springs(ys_scene* s, int mesh, const float* d_k, const float* d_L);
/* Adjoint of `steps` substeps of one FastGridCloth mesh against static
 * obstacles (self-collision off), checkpointing the scene state every
 * `checkpoint_every` substeps and replaying one segment at a time in the
 * reverse pass.  The rollout starts from the scene's state at creation. */
ys_status ys_adjoint_create(ys_adjoint** out, ys_scene* s, int mesh, uint32_t steps, uint32_t checkpoint_every);
ys_status ys_adjoint_destroy(ys_adjoint* a);
uint32_t ys_adjoint_num_springs(ys_adjoint* a);
/* Per-spring stiffness, rest length and the cloth's initial velocity (device
 * pointers; NULL keeps the current value). */
ys_status ys_adjoint_set_params(ys_adjoint* a, const float* d_k, const float* d_L, const float* d_v0);
/* Forward rollout; the cloth's final positions (3 floats per vertex) into d_xT. */
ys_status ys_adjoint_forward(ys_adjoint* a, float* d_xT);
/* dL/dx_T in; dL/dk, dL/dL (per spring) and dL/dv0 (3 floats per vertex) out. */
ys_status ys_adjoint_backward(ys_adjoint* a, const float* d_dLdx, float* d_gk, float* d_gL, float* d_gv0);
/* Arithmetic of the rollout and its reverse pass: 32 (default; the fused
 * substep's binary32 arithmetic, bit-identical to the scene's own steps) or
 * 64 (binary64 throughout, for gradients that must agree with FP64 finite
 * differences; needs static obstacles, keeps at most 16 contacts per vertex
 * and step, YS_ERR_CAPACITY beyond; the scene's own state is not advanced).
 * The float entry points above then widen their inputs and round their
 * outputs; the _f64 ones below take and give binary64 (device pointers,
 * same layouts). */
ys_status ys_adjoint_set_precision(ys_adjoint* a, int bits);
ys_status ys_adjoint_set_params_f64(ys_adjoint* a, const double* d_k, const double* d_L, const double* d_v0);
ys_status ys_adjoint_forward_f64(ys_adjoint* a, double* d_xT);
ys_status ys_adjoint_backward_f64(ys_adjoint* a, const double* d_dLdx, double* d_gk, double* d_gL, double* d_gv0);

/* ---- Standalone LBVH over one triangle soup (BVH<CUDA,PR,LINEAR,TRIANGLE>,
 * bvh.hpp:141-2308).  Device pointers; x / v packed xyz floats. ---------- */
ys_status ys_lbvh_create(ys_lbvh** out, uint32_t max_prims, int device, void* stream);
ys_status ys_lbvh_destroy(ys_lbvh* t);
/* Split of a run of equal Morton codes in the next builds.  0 (default): the
 * reference's midpoint split (findSplit, src/metal/bvh.metal:197-223), the
 * reference's tree node for node.  With three or more equal codes that tree
 * is inconsistent with determineRange's ordering: a node can be the child of
 * two internal nodes or of none, so a query reports some leaves twice and
 * never reaches others, as the reference does.  1: split by the (code,
 * index) key determineRange already orders by, so every node has one parent
 * and a query reports every overlapping leaf exactly once. */
ys_status ys_lbvh_set_split(ys_lbvh* t, int consistent);
/* Builder of the next builds (YS_BUILD_KARRAS, the default, or
 * YS_BUILD_APETREI; the Karras split option does not apply to Apetrei). */
ys_status ys_lbvh_set_builder(ys_lbvh* t, int builder);
/* build(): scene box, Morton, radix sort, Karras, leaves, bottom-up
 * (bvh.hpp:1194-1301). */
ys_status ys_lbvh_build(ys_lbvh* t, const float* d_x, uint32_t num_vertices, const uint32_t* d_facets,
                        uint32_t num_facets);
/* refit() / refitSwept(dt) (bvh.hpp:1555-1606, 1100-1115). */
ys_status ys_lbvh_refit(ys_lbvh* t, const float* d_x, const float* d_v, float dt, int swept);
/* queryPoints (bvh.hpp:1803-1841): (point, triangle) pairs for every query
 * point whose box [p - margin, p + margin] overlaps a leaf; self = skip
 * triangles containing the point.  *d_count receives the candidate count
 * (pairs beyond cap are counted, not written).  Pair order is unspecified:
 * from 2^21 query points the points are visited in their Morton order, with
 * order buffers (12 B per point plus sort scratch) kept by the tree. */
ys_status ys_lbvh_query(ys_lbvh* t, const float* d_qx, uint32_t num_queries, float margin, int self,
                        uint32_t* d_pairs, uint64_t cap, unsigned long long* d_count);
/* Device pointers of the tree arrays (nodes, parents, codes, indices). */
ys_status ys_lbvh_arrays(ys_lbvh* t, void** nodes, int32_t** parent, uint32_t** codes, uint32_t** idx,
                         uint32_t* num_prims);

/* ---- Face-face spatial-hash broad phase (SpatialHashing<METAL>::detectCollisions,
 * include/sim/spatial_hash.hpp:880-960; src/metal/spatialhashing.metal:64-478):
 * bounding spheres, a grid of cell 2*maxR + margin, a home and up to 7
 * phantom cells per face, per-cell home-home and home-phantom pairs with the
 * reference's marking dedup and sphere cull, 6 rows per surviving pair.  The
 * rows are those of the reference as a multiset (emission order differs).
 * Inputs are the packed scene (Scene::pack): positions (packed xyz), vertex
 * offsets per mesh (num_meshes + 1), facets with mesh-local vertex ids, face
 * offsets per mesh (num_meshes + 1), behaviour and collider kind per mesh.
 * Device pointers; asynchronous on the stream; no host synchronisation. */
typedef struct ys_shff ys_shff;
ys_status ys_shff_create(ys_shff** out, uint32_t max_faces, int device, void* stream);
ys_status ys_shff_destroy(ys_shff* h);
/* Rows (BroadCollision layout, 32 B) into d_rows[0, cap), which must be
 * 16-byte aligned; *d_count receives the number of rows (rows beyond cap are
 * counted, not written). */
ys_status ys_shff_detect(ys_shff* h, const float* d_x, uint32_t num_vertices, const uint32_t* d_state_off,
                         const uint32_t* d_facets, const uint32_t* d_facet_off, uint32_t num_faces,
                         const uint32_t* d_behaviors, const uint32_t* d_shapes, uint32_t num_meshes, float margin,
                         int enable_self, void* d_rows, uint64_t cap, unsigned long long* d_count);
/* Entries, cells, candidate pairs and grid resolution of the last detect
 * (the reference's LastRunStats, spatial_hash.hpp:183-208); synchronises. */
ys_status ys_shff_stats(ys_shff* h, uint32_t out6[6]);

/* ---- Uniform-grid spatial-hash broad phase, point vs triangle (the
 * spatial-hash family of the reference: SpatialHashing<METAL>::detectCollisions,
 * spatial_hash.hpp:880-960, and CpuSpatialHash, spatial_hash.hpp:1547-2016).
 * Its candidate set equals ys_lbvh_query's under the same inclusive AABB test.
 * Device pointers; x packed xyz floats. ------------------------------------ */
/* max_entries (cell entries of a build) is capped at 2^28 - 2; a build that
 * needs more fails with YS_ERR_CAPACITY. */
ys_status ys_shash_create(ys_shash** out, uint32_t max_tris, uint32_t max_entries, int device, void* stream);
ys_status ys_shash_destroy(ys_shash* h);
/* Bin every triangle's AABB into the grid cells (edge `cell`) it overlaps. */
ys_status ys_shash_build(ys_shash* h, const float* d_x, const uint32_t* d_facets, uint32_t num_facets, float cell);
/* (point, triangle) pairs whose boxes [p - margin, p + margin] and triangle
 * AABB overlap; requires cell >= 2 * margin.  Pair order is unspecified:
 * from 2^23 query points the points are visited in their Morton order. */
ys_status ys_shash_query(ys_shash* h, const float* d_qx, uint32_t num_queries, float margin, uint32_t* d_pairs,
                         uint64_t cap, unsigned long long* d_count);
/* Cell entries of the last build and triangles too large for the grid. */
ys_status ys_shash_entries(ys_shash* h, uint32_t* n_entries, uint32_t* n_oversized);

/* ---- Analytic narrow phase (BruteForce::narrowAnalytic,
 * include/sim/bruteforce.hpp:245-309; narrow_pt_analytic,
 * src/metal/bruteforce.metal:236-499): for each (cloth mesh, collider mesh)
 * pair, every vertex of the cloth against the collider's shape, the segment
 * x_prev -> x mapped into the shape's frame through its previous and current
 * pose.  A contact is appended in NarrowCollision layout (48 B: (vertex, 0),
 * (cloth, collider), normal and the signed distance of x, behaviours,
 * (YS_COLLIDER_MESH, kind)) when the distance is below radius + thickness +
 * the pair's rotation margin.  Host arrays: state_off (num_meshes + 1
 * vertex offsets), behaviors (num_meshes), shapes (num_shapes), pairs
 * (num_pairs x 2: cloth mesh index, collider mesh index, resolved to the
 * shape whose obj_index matches; pairs without one, or whose shape is not
 * collidable, are skipped).  Device arrays: d_x, d_xprev (packed xyz of all
 * meshes), d_out, d_count.  *d_count is incremented, not reset (the triangle
 * narrow phase fills the same buffer first); contacts beyond cap are counted,
 * not written.  Asynchronous on stream; allocates nothing. */
ys_status ys_narrow_analytic(const float* d_x, const float* d_xprev, const uint32_t* state_off,
                             const uint32_t* behaviors, uint32_t num_meshes, const ys_analytic_shape* shapes,
                             uint32_t num_shapes, const uint32_t* pairs, uint32_t num_pairs, float radius,
                             float thickness, void* d_out, uint64_t cap, unsigned long long* d_count, void* stream);

/* Standalone primitives used by the build. */
ys_status ys_morton_codes(const float* d_x, uint32_t num_vertices, const uint32_t* d_facets, uint32_t num_facets,
                          uint32_t* d_codes, uint32_t* d_idx, void* stream);
/* Stable LSD radix sort of (key, value) pairs, 8-bit digits, bits
 * [0, 32) (RadixSorter<METAL>::sort, spatial_hash.hpp:48-70). d_scratch of
 * ys_radix_sort_scratch_bytes(n) bytes. */
size_t ys_radix_sort_scratch_bytes(uint32_t n);
ys_status ys_radix_sort_pairs(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, void* d_scratch, void* stream);
/* The same sort for callers that cannot allocate device memory: code running
 * under CUDA-graph capture or in an allocation-free real-time loop, hosts
 * whose device memory belongs to another allocator, plugins that must not
 * grow the process's device footprint.  It calls no cudaMalloc / cudaFree and
 * no allocating library routine; its scratch is a fixed 8,651,776-byte
 * __device__ array that every GPU loading this library holds until exit.
 * At most 1,048,576 pairs (larger n returns YS_ERR_CAPACITY).  The first call
 * on a device looks up that array's device address, so make it before any
 * stream capture; after a device reset (cudaDeviceReset) the device has a new
 * context, and the first call in it looks the address up again, so make that
 * one before any capture too.  All calls share the one array: calls that overlap on the
 * GPU (different streams or threads without ordering) race.  Asynchronous on
 * `stream`.  Has no counterpart in the reference. */
ys_status ys_radix_sort_pairs_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* YSIM_B200_H */
