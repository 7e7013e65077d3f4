/*
 * br_b200.h — C ABI of the B200 (sm_100a) kinematics / LM-IK library (libbr_b200.so).
 *
 * Plain pointers and sizes only.  Every array argument is DEVICE memory unless
 * its comment says "host".  All float data is float32; poses are stored as
 * [tx, ty, tz, qx, qy, qz, qw] (scalar-last quaternion) and tangents as
 * [vx, vy, vz, wx, wy, wz], exactly as in BetterRobot
 * (src/better_robot/lie/_torch_native_backend.py:7-9).
 *
 * Every entry point enqueues work on `stream` (a cudaStream_t, NULL = legacy
 * default stream), does not synchronise, allocates no memory and returns a
 * status: BR_OK, a negative BR_E* argument error, or a positive cudaError_t.
 *
 * Which reference interface each entry point replaces is given beside it
 * (paths relative to BetterRobot's repository).
 */
#ifndef BR_B200_H
#define BR_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define BR_API __attribute__((visibility("default")))
#else
#define BR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define BR_OK 0
#define BR_EINVAL (-1)      /* null pointer, negative size, bad enum            */
#define BR_ETOOBIG (-2)     /* njoints > 64, nv > 64, more than 64 targets ...   */
#define BR_EALIGN (-3)      /* a pointer is not 4-byte (float) aligned           */

/* ---- limits ---------------------------------------------------------- */
#define BR_MAX_JOINTS 64    /* support sets are 64-bit masks                     */
#define BR_MAX_NV 64
#define BR_MAX_NQ 128
#define BR_MAX_TARGETS 64   /* frames (or joints) per Jacobian launch            */

/* ---- joint kinds in the tree table ----------------------------------- */
#define BR_JOINT_FIXED 0        /* universe, fixed                                */
#define BR_JOINT_REVOLUTE 1     /* revolute_rx/ry/rz/unaligned: rotation about axis */
#define BR_JOINT_PRISMATIC 2    /* prismatic_px/py/pz/unaligned: translation along axis */
#define BR_JOINT_FREE_FLYER 3   /* nq = 7 [t, quat], nv = 6, transform = normalize(q) */
#define BR_JOINT_SPHERICAL 4    /* nq = 4 quat, nv = 3: rotation normalize(q) (spherical.py:22-32) */
#define BR_JOINT_PLANAR 5       /* nq = 4 [x, y, cos, sin], nv = 3 (planar.py:20-41)          */
#define BR_JOINT_REVOLUTE_UNBOUNDED 6 /* nq = 2 [cos, sin], nv = 1: rotation by atan2 about axis
                                         (revolute.py:192-243)                                */
#define BR_JOINT_TRANSLATION 7  /* nq = nv = 3: translation by q (translation.py:19-23)       */

/* ---- Jacobian reference frames (kinematics/__init__.py:24-37) --------- */
#define BR_REF_WORLD 0
#define BR_REF_LOCAL_WORLD_ALIGNED 1
#define BR_REF_LOCAL 2

/*
 * Device-resident description of one kinematic tree ("tree table"), packed
 * once per Model by the host (betterrobot_b200/tree.py).  Joint j's parent
 * precedes it; joint 0 is the universe.  Replaces the per-joint Python
 * dispatch over model.joint_models / model.topo_order
 * (src/better_robot/kinematics/forward.py:110-129).
 */
typedef struct br_tree {
    int32_t njoints, nq, nv, nframes;
    int32_t rounds;           /* ceil(log2(max joint depth)): pointer-jumping rounds */
    int32_t kinds;            /* bit k set if some joint has kind BR_JOINT_k (the LM picks its
                                 kernel variant from it); the FK adjoint and trajectory
                                 optimisation reject a mask of 0                              */
    int32_t dof_entries;      /* sum over tangent columns of (depth in the DOF tree + 1): the
                                 LM's J^T J storage; 0 = not given (dense nv (nv + 1) / 2) */
    int32_t dof_depth;        /* 1 + deepest DOF-tree depth; 0 = not given (nv)            */
    const int32_t* parent;          /* [njoints]   -1 for the universe            */
    const int32_t* jtype;           /* [njoints]   BR_JOINT_*                      */
    const int32_t* idx_q;           /* [njoints]                                   */
    const int32_t* idx_v;           /* [njoints]                                   */
    const float* axis;              /* [njoints*4] local axis (x, y, z, 0)         */
    const float* placement;         /* [njoints*8] parent->joint SE3 + pad         */
    const uint64_t* support;        /* [njoints]   bit k: joint k is ancestor-or-self */
    const int32_t* frame_parent;    /* [nframes]                                   */
    const float* frame_placement;   /* [nframes*8]                                 */
    const int32_t* col_joint;       /* [nv]        joint owning tangent column c   */
    const int32_t* col_kind;        /* [nv]        0 rotation about, 1 translation along col_axis */
    const float* col_axis;          /* [nv*4]      column axis in its joint's frame */
    const float* lower;             /* [nq]        position limits (+-inf allowed) */
    const float* upper;             /* [nq]                                        */
    const uint32_t* dof_sched;      /* level schedule of the LM's J^T J factorization
                                       (br_dof_schedule, copied to the device); required by
                                       br_lm_solve / br_lm_solve_noalloc (BR_EINVAL if NULL),
                                       unused by the other entry points                      */
} br_tree_t;

/*
 * Level schedule for the LM's factorization of J^T J + damp I over the DOF tree
 * (tangent column c's parent is the previous column of its joint, or the last
 * column of the nearest ancestor joint with columns; dof_parent[c] < c, -1 at a
 * root).  The matrix is stored one row per DOF over its ancestors by depth; DOFs
 * are eliminated leaves first, and all DOFs of one height in the DOF tree (0 at a
 * leaf, 1 + the children's maximum above) at once: no two of them is an ancestor of
 * the other, so within a level the rows read and the rows written are disjoint.  An
 * entry that several DOFs of one level update (a pair of common ancestors) is one
 * task that sums their contributions in a fixed order, so the result does not depend
 * on scheduling.  The right-hand side rides along as one extra slot per DOF (forward
 * substitution inside the factorization).
 *
 * Layout (uint32 words): [0] levels, [1] tasks, [2] extra contributions, [3] 1 + the
 * deepest DOF depth, [4 .. 4 + levels] first task of each level (the last = tasks),
 * then at word toff = roundup(5 + levels, 4) the tasks, 4 words each:
 *   {dst | (n_extra << 16), a | (b << 16), k | (first_extra << 16), f}
 *   dst -= m[a] * m[b] / (pivot_k + damp), then the same for each extra contribution;
 *   f = c + 1 when the task is the last update of DOF c's diagonal (its pivot is then
 *   final), else 0,
 * then at toff + 4 * tasks the extra contributions, 2 words each: {a | (b << 16), k}.
 * Offsets index the packed rows (row c starts at sum_{c' < c} (depth(c') + 1), its
 * diagonal at depth(c)) followed by the nv right-hand-side slots.
 *
 * Writes the schedule to `out` (HOST, `capacity` words) when it fits and returns
 * the number of words it needs, or BR_EINVAL (bad dof_parent) / BR_ETOOBIG (more
 * than 65,535 packed offsets or extra contributions).  Host-only: no device work.
 */
BR_API int64_t br_dof_schedule(const int32_t* dof_parent, int32_t nv, uint32_t* out, int64_t capacity);

/*
 * Forward kinematics for `batch` configurations q[batch, nq].
 * Outputs (each may be NULL): joint_pose_world[batch, njoints, 7] (oMi),
 * joint_pose_local[batch, njoints, 7] (liMi), frame_pose_world[batch, n_frames, 7]
 * for the frame ids in `frame_ids` (HOST array of n_frames <= 64 ids).
 * Replaces KinematicsOps.forward_kinematics (src/better_robot/backends/protocol.py:58-62,
 * implemented by src/better_robot/kinematics/forward.py:73-135) and
 * update_frame_placements (forward.py:194-219).
 */
BR_API int br_forward_kinematics(const br_tree_t* tree, const float* q, int64_t batch,
                          float* joint_pose_world, float* joint_pose_local,
                          const int32_t* frame_ids, int32_t n_frames, float* frame_pose_world,
                          void* stream);

/*
 * Fused FK + frame Jacobians straight from q[batch, nq]: for each id in the HOST
 * array `targets` (n_targets <= 64; id >= 0 is a frame id, id < 0 means joint
 * (-id - 1) with identity placement) writes jacobians[batch, n_targets, 6, nv] in
 * reference frame `reference` (BR_REF_*), and if non-NULL target_pose_world
 * [batch, n_targets, 7].  Replaces forward_kinematics(..., compute_frames=True)
 * followed by get_frame_jacobian per frame (src/better_robot/kinematics/jacobian.py:129-227).
 * batch == 0 launches nothing and accepts NULL buffers.  A J block above 16 KB per
 * configuration is staged and stored in pieces of an even number of targets.
 */
BR_API int br_frame_jacobians(const br_tree_t* tree, const float* q, int64_t batch,
                       const int32_t* targets, int32_t n_targets, int32_t reference,
                       float* target_pose_world, float* jacobians, void* stream);

/*
 * Frame (or joint) Jacobians from already computed world joint placements
 * joint_pose_world[batch, njoints, 7] (Data.joint_pose_world), same target
 * encoding and output layout as br_frame_jacobians.  Replaces get_frame_jacobian
 * on a populated Data (jacobian.py:129-227) and, with targets = all joints and
 * BR_REF_WORLD, compute_joint_jacobians (jacobian.py:30-97, protocol.py:64-68).
 * batch == 0 launches nothing and accepts NULL buffers.
 */
BR_API int br_frame_jacobians_from_poses(const br_tree_t* tree, const float* joint_pose_world, int64_t batch,
                                  const int32_t* targets, int32_t n_targets, int32_t reference,
                                  float* jacobians, void* stream);

/* ==== batched Levenberg-Marquardt / Gauss-Newton IK ===================== */
#define BR_MAX_IK_CLASSES 8     /* distinct robots in one launch                   */
#define BR_MAX_IK_TARGETS 8     /* pose targets per problem                        */
#define BR_LM_SCRATCH_BYTES 16  /* device scratch br_lm_solve needs (work queue)   */
#define BR_OPT_LM 0
#define BR_OPT_GN 1
#define BR_TARGET_POSE 0        /* PoseResidual: 6 rows (residuals/pose.py:58-103)            */
#define BR_TARGET_POSITION 1    /* PositionResidual: 3 rows (pose.py:107-141), weight pos_weight */
#define BR_TARGET_ORIENTATION 2 /* OrientationResidual: 3 rows (pose.py:144-195), weight ori_weight */
#define BR_KERNEL_L2 0          /* robust kernels of OptimizerConfig.kernel (tasks/ik.py:116-133) */
#define BR_KERNEL_HUBER 1       /* w(s) = 1 if s <= d^2 else d / sqrt(s)                          */
#define BR_KERNEL_CAUCHY 2      /* w(s) = 1 / (1 + s / c^2)                                       */
#define BR_KERNEL_TUKEY 3       /* w(s) = max(1 - s / c^2, 0)^2                                   */
#define BR_IK_CONVERGED 0       /* status & 0xff                                   */
#define BR_IK_MAXITER 1
#define BR_IK_FLAG_NONFINITE 1  /* (status >> 8) bits: a non-finite cost was seen   */
#define BR_IK_FLAG_REGULARIZED 2 /* the LDL^T needed extra diagonal damping          */
#define BR_IK_FLAG_BADTREE 4    /* tree's dof_entries / dof_depth below its DOF tree: not solved */

/* Solver settings: LevenbergMarquardt(lam0, factor, tol) with Adaptive damping
 * bounds [lam_min, lam_max] (optim/strategies/adaptive.py:19-25), GaussNewton eps,
 * and the solve_ik cost weights (tasks/ik.py:38-48; limit/rest are the CostStack
 * item weights). */
typedef struct br_ik_settings {
    float lam0, factor, tol, lam_min, lam_max, gn_eps;
    float pos_weight, ori_weight, limit_weight, rest_weight;
    int32_t max_iter;
    int32_t optimizer;          /* BR_OPT_LM or BR_OPT_GN                          */
    int32_t kernel;             /* BR_KERNEL_*: IRLS row weights (levenberg_marquardt.py:27-44) */
    float kernel_param;         /* Huber delta / Cauchy c / Tukey c (optim/kernels/*.py)      */
    int32_t precision;          /* BR_PREC_*: arithmetic of the Jacobian, J^T J, J^T r and the
                                   factorization (the iterate, FK, residual and cost are float64
                                   in both)                                                   */
} br_ik_settings_t;
#define BR_PREC_F32 0           /* float32 normal equations (the default, fastest)            */
#define BR_PREC_F64 1           /* float64 normal equations: the float64 reference's iterates */

/* A packed batch of independent IK problems over up to 8 robot classes. */
typedef struct br_ik_batch {
    int32_t n_problems, max_targets, n_classes, n_items;
    const br_tree_t* trees;     /* HOST array [n_classes] (its tables live on the device) */
    const int32_t* team_size;   /* HOST array [n_classes]: lanes per problem; must be 32 */
    const int32_t* items;       /* [n_items*3] work items: first slot in order[], count <= 32/team, class */
    const int32_t* order;       /* [n_problems] problem index of each slot          */
    const int32_t* n_targets;   /* [n_problems] 1..max_targets                       */
    const int32_t* frames;      /* [n_problems*max_targets] frame ids of the class  */
    const float* targets;       /* [n_problems*max_targets*7] target poses          */
    const int64_t* q_offset;    /* [n_problems] float offset of the problem's q     */
    const float* x0;            /* packed initial configurations                    */
    const float* q_rest;        /* packed rest configurations (RestResidual q_rest) */
    const int64_t* r_offset;    /* [n_problems] float offset of the problem's stacked residual
                                   (target rows, 2*nq limit rows, nv rest rows) in result.residual;
                                   rows of a term whose weight is 0 are not written; may be NULL */
    const int32_t* target_kind; /* [n_problems*max_targets] BR_TARGET_*; NULL = every target a pose */
} br_ik_batch_t;

typedef struct br_ik_result {
    float* x;                   /* packed solutions, same offsets as x0             */
    int32_t* iters;             /* [n_problems] completed iterations (SolverState.iters) */
    int32_t* status;            /* [n_problems] BR_IK_* | flags << 8                */
    float* cost;                /* [n_problems] final 0.5 |r|^2                     */
    float* residual;            /* packed final stacked residual (CostStack order:
                                   pose targets, limits, rest); NULL = not written */
} br_ik_result_t;

/*
 * Solve every problem of `batch` in one persistent launch (one team of lanes per
 * problem, see lm_solve.cu).  `scratch` is caller-provided device memory of at
 * least BR_LM_SCRATCH_BYTES; the entry point zeroes it on `stream` before the
 * launch.  Replaces solve_ik (src/better_robot/tasks/ik.py:150-266) called once
 * per problem, i.e. LevenbergMarquardt.minimize / GaussNewton.minimize
 * (optim/optimizers/levenberg_marquardt.py:61-135, gauss_newton.py:27-76) over
 * the pose + limit + rest CostStack.  Every class tree must carry its level schedule
 * (br_tree_t.dof_sched); a schedule whose offsets do not fit the tree's DOF tree makes
 * the class's problems return BR_IK_FLAG_BADTREE.
 */
BR_API int br_lm_solve(const br_ik_batch_t* batch, const br_ik_settings_t* settings, br_ik_result_t* result,
                       int32_t warps_per_cta, void* scratch, int64_t scratch_bytes, void* stream);

/*
 * Same solve as br_lm_solve for callers that cannot allocate device memory at all
 * (e.g. a robot controller's real-time loop, where cudaMalloc may block and
 * serialise the device, or a host with no CUDA allocator that only owns its
 * inputs and outputs).  The work-queue scratch comes from a static device array
 * of BR_LM_NOALLOC_SCRATCH_BYTES inside the library (one per device, kept until
 * the process exits) instead of a caller pointer; a launch needing more than that
 * returns BR_ETOOBIG.  The first call on each device looks up the array's device
 * address and should be made before any stream capture; the address is kept, so a
 * cudaDeviceReset between calls is not supported.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.  No
 * counterpart in the reference (BetterRobot has no native code).
 */
#define BR_LM_NOALLOC_SCRATCH_BYTES 256
BR_API int br_lm_solve_noalloc(const br_ik_batch_t* batch, const br_ik_settings_t* settings,
                               br_ik_result_t* result, int32_t warps_per_cta, void* stream);

/* Shared-memory floats one problem of `tree` with `max_targets` targets needs in the
 * float32 variant (BR_PREC_F32; the float64 variant needs more, and the solve entry
 * points size their launches themselves). No reference counterpart. */
BR_API int64_t br_lm_team_floats(const br_tree_t* tree, int32_t max_targets);

/* ==== pose loss through FK and its adjoint ================================ */
/*
 * loss[b] = sum_f w_f |log(T_f^-1 * oMf_f(q_b))|^2 for the frames in the HOST
 * array frame_ids (n_frames <= 64), targets[b, f, 7], weights[f] (or
 * weights[b, f] if weights_per_config).  If joint_pose_world is non-NULL the
 * world joint placements [batch, njoints, 7] are stored for the backward pass
 * ("store" mode).  The reference evaluates this loss with its per-op torch FK
 * (src/better_robot/kinematics/forward.py:73-135, lie/se3.py log/compose).
 */
BR_API int br_pose_loss(const br_tree_t* tree, const float* q, int64_t batch, const int32_t* frame_ids,
                        int32_t n_frames, const float* targets, const float* weights, int32_t weights_per_config,
                        float* loss, float* joint_pose_world, void* stream);

/*
 * Adjoint of br_pose_loss: grad_q[b, :] = grad_loss[b] * dloss[b]/dq (raw q of every
 * joint kind: free-flyer and spherical quaternion components, planar [x, y, cos, sin],
 * unbounded revolute [cos, sin] included).  joint_pose_world from the
 * forward pass, or NULL to recompute FK from q ("recompute" mode).  Replaces
 * torch autograd's backward through the reference FK tape
 * (forward.py:79-81 builds that tape on purpose).
 */
BR_API int br_pose_loss_backward(const br_tree_t* tree, const float* q, const float* joint_pose_world,
                                 int64_t batch, const int32_t* frame_ids, int32_t n_frames, const float* targets,
                                 const float* weights, int32_t weights_per_config, const float* grad_loss,
                                 float* grad_q, void* stream);

/* ==== batched trajectory optimisation (Gauss-Newton / LM) ================ */
#define BR_MAX_TRAJ_KNOTS 128
#define BR_MAX_TRAJ_NV 64

/* Cost stack weights (CostStack item weights) and solver settings.  Terms with
 * weight 0 are left out. */
typedef struct br_traj_settings {
    float dt;                   /* knot spacing of the acceleration residual        */
    float w_goal, w_start;      /* PoseResidual at knot T-1 / knot 0                */
    float w_accel;              /* AccelerationResidual                             */
    float w_limit;              /* JointPositionLimit at every knot                 */
    float w_ref;                /* ReferenceTrajectoryResidual (toward x_ref)       */
    float tol, gn_eps, lam0, factor, lam_min, lam_max;
    int32_t max_iter;
    int32_t optimizer;          /* BR_OPT_GN or BR_OPT_LM                           */
} br_traj_settings_t;

/*
 * Solve n_traj independent trajectories of `knots` configurations each, one CTA
 * of 128 threads per trajectory, with the Newton step in nested-dissection order
 * (per-DOF pentadiagonal interior, dense Schur complement on the end knots).  x0 / x_ref / x
 * are [n_traj, knots, nq] (x_ref NULL = x0), goal / start are [n_traj, 7] poses of
 * frame `frame_id` (start may be NULL).  goal_grad (NULL or [n_traj, 6]) receives
 * d(final cost)/d(eps) for the goal perturbed as T_goal * exp(eps).  Every joint kind
 * (knot differences and the retraction through Model.difference / Model.integrate);
 * nv <= BR_MAX_TRAJ_NV; BR_ETOOBIG when one trajectory's working set (about
 * 8 (7 knots nv + 2 knots nq + 2 nv^2) bytes) exceeds the device's shared memory per
 * CTA (e.g. the 36-DOF humanoid fits up to 64 knots).
 * Replaces solve_trajopt with the knot parameterisation and its dense LM / GN
 * (src/better_robot/tasks/trajopt.py:84-230) on the goal / start / acceleration /
 * limit / reference-trajectory stack.
 */
BR_API int br_trajopt_solve(const br_tree_t* tree, int32_t frame_id, int64_t n_traj, int32_t knots,
                            const float* x0, const float* x_ref, const float* goal, const float* start,
                            const br_traj_settings_t* settings, float* x, int32_t* iters, int32_t* status,
                            float* cost, float* goal_grad, void* stream);

/* ==== configuration-space retraction / difference ======================== */
#define BR_OP_INTEGRATE 0   /* out[B, nq] = a (+) b,  a = q [B, nq], b = v [B, nv]      */
#define BR_OP_DIFFERENCE 1  /* out[B, nv] = b (-) a,  a = q0 [B, nq], b = q1 [B, nq]    */

/*
 * Batched Model.integrate / Model.difference
 * (src/better_robot/data_model/model.py:160-190): per joint q + v / q1 - q0, and for
 * a free-flyer normalize(q exp(v)) / log(q0^-1 q1).  active_joints is a DEVICE array
 * of the n_active joint ids with nq > 0.
 */
BR_API int br_configuration_op(const br_tree_t* tree, const int32_t* active_joints, int32_t n_active, int32_t op,
                               const float* a, const float* b, int64_t batch, float* out, void* stream);

/* ==== batched SE3 / SO3 primitives (the LieOps seam) ====================== */
/*
 * Replaces the per-op LieOps protocol (src/better_robot/backends/protocol.py:27-51)
 * as implemented by src/better_robot/lie/_torch_native_backend.py and the SE3 right
 * Jacobians of src/better_robot/lie/tangents.py:184-207.  Element sizes (floats):
 */
#define BR_LIE_SE3_COMPOSE 0      /* a 7, b 7 -> 7        se3_compose     :237-246 */
#define BR_LIE_SE3_INVERSE 1      /* a 7      -> 7        se3_inverse     :249-255 */
#define BR_LIE_SE3_LOG 2          /* a 7      -> 6 [v,w]  se3_log         :289-310 */
#define BR_LIE_SE3_EXP 3          /* a 6      -> 7        se3_exp         :258-286 */
#define BR_LIE_SE3_ACT 4          /* a 7, b 3 -> 3        se3_act         :313-315 */
#define BR_LIE_SE3_ADJOINT 5      /* a 7      -> 36 (6x6 row-major)  se3_adjoint :318-328 */
#define BR_LIE_SE3_ADJOINT_INV 6  /* a 7      -> 36       se3_adjoint_inv :331-342 */
#define BR_LIE_SE3_NORMALIZE 7    /* a 7      -> 7        se3_normalize   :358-361 */
#define BR_LIE_SO3_COMPOSE 8      /* a 4, b 4 -> 4        so3_compose     :134-135 */
#define BR_LIE_SO3_INVERSE 9      /* a 4      -> 4        so3_inverse     :138-141 */
#define BR_LIE_SO3_LOG 10         /* a 4      -> 3        so3_log         :162-183 */
#define BR_LIE_SO3_EXP 11         /* a 3      -> 4        so3_exp         :144-159 */
#define BR_LIE_SO3_ACT 12         /* a 4, b 3 -> 3        so3_act         :186-199 */
#define BR_LIE_SO3_TO_MATRIX 13   /* a 4      -> 9 (3x3 row-major)   so3_to_matrix :210-211 */
#define BR_LIE_SO3_FROM_MATRIX 14 /* a 9      -> 4        so3_from_matrix :206-207 */
#define BR_LIE_SO3_NORMALIZE 15   /* a 4      -> 4        so3_normalize   :202-203 */
#define BR_LIE_SE3_JR 16          /* a 6      -> 36       tangents.right_jacobian_se3     :184-201 */
#define BR_LIE_SE3_JR_INV 17      /* a 6      -> 36       tangents.right_jacobian_inv_se3 :204-207 */

/*
 * out[i] = op(a[i], b[i]) for i < n, float32, contiguous records.  na and nb are n or
 * 1 (1 broadcasts that operand); b is ignored by unary ops.  Device pointers.
 */
BR_API int br_lie_op(int32_t op, const float* a, int64_t na, const float* b, int64_t nb, float* out, int64_t n,
                     void* stream);
/* Floats per element of a, b (0 for unary ops) and out for op; host only. */
BR_API int br_lie_op_sizes(int32_t op, int32_t* a_floats, int32_t* b_floats, int32_t* out_floats);

/* Library build information (for logging): returns a static string. */
BR_API const char* br_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BR_B200_H */
