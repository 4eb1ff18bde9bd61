/*
 * sf.h — C ABI of the B200 (sm_100a) Shatterforge physics path.
 *
 * The reference engine is a wasm32 Rust module driven through a handful of `extern "C"` exports on one static
 * world (src/lib.rs:3613-4057). This header is the drop-in boundary for its two hot-path entry points:
 *
 *   sf_world_step        replaces `pub extern "C" fn step(dt: f32)`               src/lib.rs:3639-3651
 *                        (the rigid part: two substeps of update_cache, build_hash, gen_contacts, prep_contacts,
 *                        the impulse iterations, pinch clamps, integrate — src/lib.rs:1769-1783)
 *   sf_structure_solve   replaces the load-path sweeps of `structural(w, dt)` and `warm_step(w)`
 *                        (sor_struct / sor_brick, src/lib.rs:1005-1079, 1268-1281)
 *   sf_structure_check   replaces the joint pass of `structural` (stress_brick, src/lib.rs:1153-1227, 1323-1339)
 *   sf_world_connectivity replaces `connectivity(w)` (conn_struct, src/lib.rs:1085-1141), which `step` runs after
 *                        the substeps and again after `structural` (src/lib.rs:3653, 3659)
 *
 * and for the read-outs the reference hands out as raw pointers (`ptr_stats`, `ptr_structs`, … src/lib.rs:4026-4057)
 * it offers copy-out readers into caller buffers. Plain pointers and sizes only; every call returns an sf_status
 * and never aborts. A world handle is not thread-safe; distinct handles are.
 *
 * Units and frames follow the reference: metres, seconds, kilograms; the lattice is 640 x 136 x 640 cells of
 * 0.5 m whose cell (x, y, z) has its centre at ((x - 320) * 0.5 + 0.25, y * 0.5 + 0.25, (z - 320) * 0.5 + 0.25)
 * (src/lib.rs:113-120, 355-357). Quaternions are (x, y, z, w).
 */
#ifndef SHATTERFORGE_SF_H
#define SHATTERFORGE_SF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t sf_status;
#define SF_OK 0
#define SF_ERR_ARG 1        /* bad argument: null pointer, out-of-lattice brick, duplicate cell, unknown id */
#define SF_ERR_CAPACITY 2   /* a device capacity was exceeded (contacts, colours); counts are in sf_stats */
#define SF_ERR_CUDA 3       /* a CUDA call failed (no device, out of memory, launch failure) */
#define SF_ERR_TIMEOUT 4    /* a bounded device wait (grid barrier) gave up; the context stays usable */
#define SF_ERR_BUDGET 5     /* the serving memory budget cannot hold the request */
#define SF_ERR_STATE 6      /* call out of order (e.g. reading contacts before any step) */
#define SF_ERR_VERIFY 7     /* a device self-check failed (improper colouring, island invariant) */

/* solve and sleep switches */
#define SF_SLEEP_BODY 0     /* per-body rest timer, src/lib.rs:1720-1734 (the reference's rule) */
#define SF_SLEEP_ISLAND 1   /* island rule of gpu/gpu_world.js:1660-1668 over the same timers */

typedef struct sf_world sf_world;

/* One independent world (scene). Static bricks sit on lattice cells; body bricks are given in local lattice
 * coordinates and turned into a compound body by setup_body (src/lib.rs:844-891) about the parent pose. */
typedef struct sf_scene_desc {
    uint32_t n_static;
    const int32_t *static_xyz;      /* 3 per brick: lattice x (0..639), y (0..135), z (0..639) */
    const uint8_t *static_mat;      /* material 1..8 (src/lib.rs:163-164) */
    const int32_t *static_sid;      /* structure id >= 0, or -1 for loose static geometry */
    const uint8_t *static_infill;   /* 1 = infill (non-bearing); glass is always infill (src/lib.rs:632) */
    uint32_t n_bodies;
    const uint32_t *body_first;     /* n_bodies + 1 prefix offsets into the body-brick arrays */
    const int32_t *body_brick_xyz;  /* 3 per body brick: local lattice cell */
    const uint8_t *body_brick_mat;
    const float *body_pose;         /* 13 per body: parent position 3, quaternion 4, velocity 3, spin 3 */
} sf_scene_desc;

typedef struct sf_world_desc {
    uint32_t n_scenes;
    const sf_scene_desc *scenes;
    int32_t structure_offset_per_scene; /* 0: structure ids are world-global as given */
} sf_world_desc;

typedef struct sf_params {
    uint32_t substeps;          /* substeps per step (reference: 2, src/lib.rs:3650) */
    uint32_t iterations;        /* impulse iterations per substep (reference: 10, src/lib.rs:1779) */
    uint32_t sleep_mode;        /* SF_SLEEP_BODY or SF_SLEEP_ISLAND */
    uint32_t pinch_kill;        /* 1: small pinched bodies are removed as the reference does (src/lib.rs:1755) */
    uint32_t max_colors;        /* manifold colour limit, <= 1024 (default 128): a body with thousands of contacts,
                                   whose chunks all conflict, needs more */
    uint32_t contact_capacity;  /* 0 = automatic (grows between steps) */
    uint32_t verify;            /* 1: check the colouring is proper every substep (SF_ERR_VERIFY on failure) */
    uint32_t solve_blocks;      /* persistent-kernel blocks per SM for the solve (0 = autotuned) */
    uint32_t manifold_chunk;    /* a body pair's contacts are solved in chunks of at most this many, 1..32 (0 or more
                                   than 32 mean 32); chunks of one pair take different colours, bounding each
                                   colour's longest chain and the contact layout's depth */
    uint32_t sor_cluster;       /* 1: a structure of at most 65,534 bricks is solved by one thread-block cluster that
                                   keeps its cells in shared memory (same potentials and sweeps); 0: always the
                                   grid-wide kernel */
    uint32_t detach_bodies;     /* spare bodies per scene for pieces that sf_structure_connect detaches (0 = none) */
    uint32_t detach_bricks;     /* spare body bricks per scene for those pieces */
    uint32_t damage;            /* 1: damage on contact in every substep (impact_damage, src/lib.rs:1602-1702);
                                   needs spare capacity */
    uint32_t reduce;            /* 1: contact reduction (gpu/gpu_world.js:834-920): a body pair with more than 32
                                   contacts keeps, per direction to the 26 neighbours of a cube cell, the contact
                                   whose point reaches furthest along it, and the deepest (ties to the later contact);
                                   the rest are neither coloured nor solved and carry no impulse. Bounds a pair's
                                   chunks, so a body resting on thousands of contacts needs few colours */
    uint32_t warm_start;        /* 1: warm start (gpu/gpu_world.js:557-576, 615-683): a contact found in the last
                                   substep's table by its key (its brick, the other side's kind and brick, its place
                                   among the brick's contacts with that brick) starts from 0.8 of that substep's
                                   normal impulse and friction (projected on its tangents, clamped to the cone),
                                   applied once before the iterations in the solve's order. The table starts over
                                   after a rebuild or a detachment moves brick ids */
    uint32_t reserved[1];
} sf_params;

typedef struct sf_stats {
    uint64_t contacts;          /* last substep */
    uint64_t manifolds;
    uint64_t ref_would_drop;    /* contacts past the reference's MAXC = 30000 (src/lib.rs:1397), per scene summed */
    uint32_t colors;            /* colours used by the last substep's manifold colouring */
    uint32_t color_rounds;      /* Jones-Plassmann rounds */
    uint32_t islands;           /* islands of awake bodies (last substep) */
    uint32_t alive, awake;      /* bodies after the last step */
    uint32_t error_word;        /* device error bits (0 = none) */
    uint64_t contact_capacity;
    double ms_last_step;        /* device time of the last sf_world_step call (CUDA events) */
    uint64_t launches;          /* kernels this world has launched (all entry points) */
    uint64_t graph_launches;    /* load-path solves replayed from a captured CUDA graph */
    uint64_t cluster_solves;    /* load-path solves run by one thread-block cluster per structure */
} sf_stats;

/* Per-phase device time of the rigid step, from CUDA events around each phase of each substep (profiling on). */
#define SF_PHASES 9             /* pose, hash, contacts, manifolds, colour, prep, solve, islands, integrate */
typedef struct sf_profile {
    double ms[SF_PHASES];
    uint64_t substeps;
    uint64_t solve_launches;
    uint64_t solve_contact_iters;   /* sum over solve launches of contacts x iterations */
    uint64_t contacts_sum;          /* sum over substeps of contacts */
    uint64_t launches;
    double gen_ms;                  /* device time of the contact-generation kernel alone (inside the contacts phase) */
    uint64_t gen_bricks;            /* sum over its launches of the bricks it visited */
} sf_profile;

typedef struct sf_solve_report {
    uint32_t structures;        /* structures solved */
    uint32_t max_sweeps_done;   /* the most sweeps any structure took */
    uint64_t brick_sweeps;      /* sum over structures of bricks x sweeps */
    double max_residual;        /* the largest final residual (reference measure: max|dphi| / max(phi, 1)) */
    double ms;                  /* device time of the solve (CUDA events) */
} sf_solve_report;

typedef struct sf_check_report {
    uint64_t joints;            /* joints evaluated */
    uint64_t over;              /* joints with ratio > 1 */
    uint64_t failed;            /* bond failures (tension / shear) */
    uint64_t crushed;           /* compressive crushes (a brick removed) */
    float max_ratio;
    double ms;
} sf_check_report;

/* ---- lifecycle */
void sf_params_default(sf_params *p);
sf_status sf_world_create(const sf_world_desc *desc, const sf_params *params, sf_world **out);
void sf_world_destroy(sf_world *w);
const char *sf_status_string(sf_status s);
const char *sf_last_error(void);
int32_t sf_version(void);

/* All of the world's device work goes to `stream` (a cudaStream_t; NULL = the world's own stream). */
sf_status sf_world_set_stream(sf_world *w, void *stream);
/* Phase timing with CUDA events (off by default; costs ten event records per substep). */
sf_status sf_set_profiling(sf_world *w, int32_t on);
sf_status sf_read_profile(sf_world *w, sf_profile *out);
sf_status sf_reset_profile(sf_world *w);
/* The launch-shape autotuner: persistent kernels' blocks per SM, chosen per size bucket (bucket b holds launches of
 * 2^b .. 2^(b+1) - 1 work items: contacts for the solve and the colouring, chunks for the load solve) by timing each
 * candidate on the bucket's first launches. These shapes never change results. Writes the chosen value per bucket
 * (-1 = not settled yet) for the first n buckets. */
#define SF_TUNE_SOLVE 0
#define SF_TUNE_COLOR 1
#define SF_TUNE_SOR 2
sf_status sf_read_tuning(sf_world *w, uint32_t which, int32_t *blocks_per_sm, uint32_t n);
/* Self-check of the device-side waits (no counterpart in the reference): one kernel waits on a flag that nothing
 * sets, through the same bounded wait the persistent kernels' grid barriers use, with a limit of limit_ms (1..2000).
 * Returns SF_ERR_TIMEOUT when the wait gave up as it should (the context stays usable), and the device time waited. */
sf_status sf_check_wait_timeout(uint32_t limit_ms, double *waited_ms);

/* ---- hot path */
/* nsteps world steps of dt each (dt clamped to [0, 1/30] as src/lib.rs:3642 does), all scenes at once. Scenes
 * whose bodies all sleep are skipped (a step leaves them unchanged), so the cost follows the awake scenes. */
sf_status sf_world_step(sf_world *w, float dt, uint32_t nsteps);
/* As sf_world_step, but only the scenes with scene_mask[scene] != 0 step (host array of n_scenes bytes); the others
 * are left exactly as they are. No counterpart in the reference (one world per wasm instance there): this is the
 * batched form's way to step a chosen subset of resident scenes in one set of launches. */
sf_status sf_world_step_scenes(sf_world *w, float dt, uint32_t nsteps, const uint8_t *scene_mask);
/* Load-path solve of one structure (>= 0) or of every structure (-1): red-black SOR with relaxation omega until
 * the reference's residual max|dphi| / max(phi, 1) < tol or max_sweeps. */
sf_status sf_structure_solve(sf_world *w, int32_t structure, float omega, float tol, uint32_t max_sweeps,
                             sf_solve_report *report);
/* The same solve for a list of structures in one persistent launch (each structure stops at its own residual).
 * Every solve starts from the stored potentials, so a solve split over several calls of k sweeps each takes the
 * same sweeps as one call. No counterpart in the reference (its structures are solved one per `structural` call);
 * this is the batched form's entry point. */
sf_status sf_structure_solve_set(sf_world *w, const int32_t *structures, uint32_t n, float omega, float tol,
                                 uint32_t max_sweeps, sf_solve_report *report);
/* ext[brick[k]] += value[k] for k in order: external loads on static bricks (the body-load term of `structural`
 * folds into ext the same way, src/lib.rs:1257-1258). */
sf_status sf_structure_add_loads(sf_world *w, uint32_t n, const uint32_t *brick, const float *value);
/* Joint checks of one structure (or -1 = all) on the current potentials; live != 0 applies fatigue, failures and
 * crushes as stress_brick does. */
sf_status sf_structure_check(sf_world *w, int32_t structure, float dt, int32_t live, sf_check_report *report);
/* Resting-body loads of `structural` (src/lib.rs:1233-1259) for the listed structures: brick positions refreshed as
 * update_cache does, each body's weight shared over the listed structures' bricks under it and the ground, summed
 * per brick in body-then-brick order into extn, then ext = 0.8 ext + 0.2 extn. */
sf_status sf_structure_loads(sf_world *w, const int32_t *structures, uint32_t n_structures);
/* The reference's per-frame load-path schedule, with this library's red-black FP64 sweeps in place of its
 * lexicographic f32 ones (the schedule's residual tests then see FP64 residuals):
 *   sf_structure_warm    warm_struct (src/lib.rs:1061-1066): a structure not yet solved gets 560 warm-up sweeps pending
 *                        and a settle timer that starts when they are done (once per structure)
 *   sf_structure_frame   one frame: the sweep loop of `structural` (src/lib.rs:1268-1281) over the listed active
 *                        structures, in order (omega 1.85; nmin sweeps by the residual of the structure's last sweep:
 *                        below 1e-4 one on every third frame, counted by (frame + structure) % 3 == 0, else none;
 *                        otherwise 1 for more than 15,000 bricks and 6 for fewer; then more while its residual is at
 *                        least 4e-4, it has done fewer than 90 and a budget of 160,000 brick-updates shared in order
 *                        is left); the joint pass of the structures that are live (settle timer <= 0 and residual
 *                        below 1.5e-3, src/lib.rs:1323-1339: fatigue, failures and crushes applied, one crush budget
 *                        of 300 for the frame); the settle timers (src/lib.rs:1334); then warm_step
 *                        (src/lib.rs:1068-1079: pending warm-up sweeps in structure order from a budget of 120,000
 *                        brick-updates, omega 1.9 while more than 60 remain, then 1.0). Only structures passed to
 *                        sf_structure_warm are swept.
 * sf_read_structure_state returns per structure its pending warm-up, solved flag, settle timer and last residual
 * (n_structures entries each, any NULL). */
typedef struct sf_frame_report {
    uint32_t sweeps;            /* structural sweeps this frame, summed over structures */
    uint32_t warm_sweeps;       /* warm-up sweeps this frame, summed over structures */
    uint64_t brick_updates;     /* bricks x sweeps, both kinds */
    double ms;                  /* device time of the frame's solves */
    uint32_t live;              /* structures whose joints were judged live this frame */
    float max_ratio;            /* the live joints' largest ratio */
    uint64_t joints, over, failed, crushed;   /* the live joint pass, as sf_check_report */
} sf_frame_report;
sf_status sf_structure_warm(sf_world *w, int32_t structure);
sf_status sf_structure_frame(sf_world *w, uint32_t frame, float dt, const int32_t *active, uint32_t n_active,
                             sf_frame_report *report);
sf_status sf_read_structure_state(sf_world *w, int32_t *warm, uint8_t *solved, float *settle, double *resid);

/* ---- connectivity and detachment (conn_struct, src/lib.rs:1085-1134; connectivity, src/lib.rs:1137-1141)
 * A structure's static bricks that no longer reach a grounded footing through intact bonds become rigid bodies: one
 * body per bonded piece, its bricks in the order of the reference's breadth-first walk (pieces seeded in brick order,
 * neighbours in the order +x, -x, +y, -y, +z, -z), set up at rest with the identity rotation (setup_body,
 * src/lib.rs:844-891), and every sleeping body within (radius + 1.5 m + its radius) of a new body is woken
 * (wake_near, src/lib.rs:925-929). A new body takes the scene's next spare body and its bricks the next spare body
 * bricks (sf_params.detach_bodies / detach_bricks); a piece that does not fit stays static and its structure stays
 * pending, as the reference retries when its body pool is full. The detached static bricks are removed (material 0,
 * potential and loads 0); their bonds, which now join body bricks, are kept.
 * sf_structure_connect runs the listed structures in the given order; sf_world_connectivity runs, in structure
 * order, every structure pending since the last call: one whose joint failed or whose brick was crushed in a joint
 * pass (sf_structure_check or sf_structure_frame with live joints), or one left pending by a piece that did not fit.
 * now / top (optional, indexed by structure id, n_structures entries) receive, for each structure walked, the bricks
 * of it still standing and its height in cells (st_now, st_top, src/lib.rs:1126-1128); other entries are untouched. */
typedef struct sf_connect_report {
    uint32_t structures;        /* structures walked */
    uint32_t pieces;            /* bodies created */
    uint32_t detached;          /* static bricks that became body bricks */
    uint32_t retry;             /* structures left pending because a piece did not fit */
    uint64_t listed;            /* static bricks of unsupported pieces read back from the GPU for the walk */
    double ms;                  /* host wall time of the call */
} sf_connect_report;
sf_status sf_structure_connect(sf_world *w, const int32_t *structures, uint32_t n, uint32_t *now, int32_t *top,
                               sf_connect_report *report);
sf_status sf_world_connectivity(sf_world *w, uint32_t *now, int32_t *top, sf_connect_report *report);
/* ---- brick removal and body splitting (remove_brick, src/lib.rs:705-718; rebuild_body, src/lib.rs:930-1002)
 * A world created with spare capacity (detach_bodies / detach_bricks) gives body bricks bonds: finalize_brick's rule
 * between face-adjacent bricks of one body (glass is infill), or the bonds a detached piece's bricks had as static
 * bricks. sf_world_remove_bricks removes static bricks (world static ids: material 0, out of the grid, their
 * structures pending a connectivity walk) and body bricks (world body-brick ids: material 0, their bodies marked).
 * sf_world_rebuild_bodies runs rebuild_body on every marked body in body order: removed bricks leave it, the rest
 * split into components bonded by intact bonds (seeded in the body's brick order, breadth first); the first stays in
 * the body, its bricks moved to the front of the body's brick range, each other takes the scene's next spare body and
 * bricks (without room for all of them the body stays whole, as the reference when its pool is full); every piece is
 * set up from its bricks' local offsets about the parent's pose and cached rotation, awake. With more than 1,500
 * bodies of the scene awake, a lone-brick piece other than steel becomes debris (removed) with probability
 * min((awake - 1500) / 2000, 0.85), drawn from h01 (src/lib.rs:341-345) of the scene's count of rebuilt bodies and
 * the brick's place in its body instead of the world's random stream. A body left with no brick dies. */
typedef struct sf_rebuild_report {
    uint32_t bodies;            /* bodies rebuilt */
    uint32_t pieces;            /* new bodies */
    uint32_t removed;           /* bricks of material 0 that left their bodies */
    uint32_t dissolved;         /* bodies that died with no brick left */
    uint32_t lone;              /* lone-brick pieces turned to debris */
    uint32_t reserved;
    double ms;                  /* host wall time of the call */
} sf_rebuild_report;
sf_status sf_world_remove_bricks(sf_world *w, const uint32_t *statics, uint32_t n_statics, const uint32_t *body_bricks,
                                 uint32_t n_body_bricks);
sf_status sf_world_rebuild_bodies(sf_world *w, sf_rebuild_report *report);
/* ---- damage on contact (impact_damage / crush_at / plough, src/lib.rs:1493-1550, 1602-1702), with sf_params.damage = 1
 * Every substep, between the contacts and prep_contacts, plough: in list order, a body driving into a static brick at
 * 2 m/s or more with momentum min(3 m / max(contacts, 3), m) vn of at least 0.35 CAPV of the brick damages it (a body
 * of more than 40 bricks: damage_brick by mom / 1.5 CAPV within 0.15..0.9) or, while the scene has a spare body and
 * brick, knocks it loose as a severed one-brick body moving at 0.75 of the body's velocity plus 2 m/s with a spin of
 * 6 rad/s in random directions (rndv on the scene's draw count); the body keeps m / (m + 1.5 MASS) of its velocity and
 * that contact and the later ones with the brick are switched off. Between the pinch clamps and integration: each contact's absorbed energy E = 1/2 jn vn0 (at least
 * 150 J at an approach speed of at least 1 m/s) is split between its bricks in proportion to 1 / EB and crushes each
 * side's bricks nearest the contact point, growing through intact bonds within the body or structure, one budget of
 * 2,500 bricks per scene and substep in contact list order; the brick a share cannot afford is cracked (its bonds
 * weakened by 0.6 E / EB of their capacity). A crushed brick is ground away with probability PULV of its material
 * (drawn from h01 of a fixed seed and the scene's draw count), else severed. Removed or severed static bricks leave
 * their structures pending a connectivity walk; bodies that lose or sever bricks are marked for
 * sf_world_rebuild_bodies. The frame then runs, as `step` does (src/lib.rs:3650-3659): sf_world_step,
 * sf_world_rebuild_bodies, sf_world_connectivity, the load-path calls, sf_world_connectivity.
 * sf_read_damage returns the counters since the last read and, per structure, whether a hit woke it (a heavy hit
 * with jn vn0 > 4,000, or a brick of it damaged: st_activate), then clears both. */
typedef struct sf_damage_report {
    uint64_t contacts;          /* candidate contacts walked */
    uint64_t crushed;           /* bricks crushed */
    uint64_t removed;           /* of them ground away */
    uint64_t severed;           /* of them severed from their neighbours */
    uint64_t cracked;           /* bricks whose bonds a leftover share weakened */
    uint64_t ploughed;          /* static bricks a small body knocked loose (plough) */
    uint64_t scraped;           /* static bricks a large body damaged in passing (plough) */
} sf_damage_report;
sf_status sf_read_damage(sf_world *w, sf_damage_report *report, uint8_t *activated);
/* body bricks' bonds (4 each: +x, +y, +z, foundation) and face neighbours (6 each, world body-brick ids) */
sf_status sf_read_body_bonds(sf_world *w, float *bond4, uint32_t *nb6);

/* ---- the debris-body load field (structural's body part, src/lib.rs:1262-1266, 1282-1365), in a world with spare
 * capacity. After the structures' frame (sf_structure_frame), per scene in body order:
 *   - a piece of 8 or more bricks none of whose bricks a contact supported in the last 10 frames (a contact from
 *     below: the ground, a static brick, or another body's brick; stamped in every substep) starts its potentials over;
 *   - a loaded piece (alive, awake, in contact, 8 or more bricks, its first brick not slug) carries the inertial load
 *     MASS (n - 1) per brick, n = |g - a| / g (at most 150), a = the change of the piece's velocity and spin over the
 *     frame (dt at least 1 ms) at the brick's position; the peak n is kept;
 *   - a loaded piece of at most 60,000 bricks whose field is not settled (residual below 2e-4 and peak below 1.5),
 *     or is and whose id in its scene plus the frame count is a multiple of 4, is swept red-black in FP64 with
 *     omega 1.8, a supporting brick resting on the ground: at least 2 sweeps, until the residual falls below 4e-4,
 *     60 sweeps or the scene's budget of 160,000 brick updates (sweeps x brick count, shared in body order) is spent;
 *   - its load time grows by dt; it is judged unless settled and off its fourth frame (settled: with 4 dt); its
 *     joints are live once loaded 0.3 s with a residual below 1e-2 (or 0.6 s), or at once above a peak of 2.5.
 *     A live over-stressed joint fatigues at the material's DUCT pace; below 8% of its capacity it fails, or, in
 *     pure compression along a near-vertical axis while the frame's 300 crushes last (counted on from crushes_used,
 *     the structures' joint pass's crushes, one budget for the call), the weaker brick is crushed. A failure or a
 *     crush marks the piece for sf_world_rebuild_bodies;
 *   - a live piece that is not loaded lets its load time run down by 2 dt.
 * The frame order of `step` (src/lib.rs:3650-3659) is then sf_world_step, sf_world_rebuild_bodies,
 * sf_world_connectivity, sf_structure_loads, sf_structure_frame, sf_bodies_frame, sf_world_connectivity.
 * sf_read_body_fields returns per body brick the f64 potential and the inertial load, and per body the last
 * residual, the peak load factor, the load time and the largest joint ratio of its last judgement (any NULL). */
typedef struct sf_bodies_report {
    uint32_t bodies;            /* pieces swept */
    uint32_t sweeps;            /* their sweeps */
    uint64_t brick_updates;     /* sweeps x brick count */
    uint32_t judged;            /* pieces whose joints were judged */
    uint32_t crushes_used;      /* the frame's crushes after this pass (structures' and pieces') */
    uint64_t joints, over, failed, crushed;   /* the judged joints, as sf_check_report */
    float max_ratio;            /* the judged joints' largest ratio */
    float reserved;
    double ms;                  /* host time of the call */
} sf_bodies_report;
sf_status sf_bodies_frame(sf_world *w, float dt, uint32_t crushes_used, sf_bodies_report *report);
sf_status sf_read_body_fields(sf_world *w, double *phi64, float *ext, double *resid, float *nmax, float *lt,
                              float *maxr);

/* per scene: static_off, n_static, body_off, body capacity, brick_off, brick capacity, bodies used, bricks used */
sf_status sf_world_scene_ranges(const sf_world *w, uint32_t scene, uint32_t out8[8]);
/* Per-structure sweeps and final residuals of the last sf_structure_solve (n_structures entries each). */
sf_status sf_read_solve_detail(sf_world *w, uint32_t *sweeps, double *resid);

/* ---- read-outs (copy into caller buffers; body and brick order is world-global, scene-major) */
typedef struct sf_world_info {
    uint32_t n_scenes, n_static, n_bodies, n_body_bricks, n_structures, n_chunks;
} sf_world_info;
sf_status sf_world_get_info(const sf_world *w, sf_world_info *info);
sf_status sf_get_stats(const sf_world *w, sf_stats *stats);
/* 13 floats per body (pos 3, quat 4, v 3, spin 3); sleep timer; flags bit0 alive, bit1 asleep. A write refreshes
 * the rotation cache and brick positions of every body whose pose it changes (sleeping ones included); bodies
 * written with their current pose keep their caches, so reading and writing back the state changes nothing. */
sf_status sf_read_bodies(sf_world *w, float *state13, float *sleep, uint8_t *flags);
sf_status sf_write_bodies(sf_world *w, const float *state13, const float *sleep, const uint8_t *flags);
/* per body: mass, 1/mass, radius, local inverse inertia 9; per body brick: local offset 3 */
sf_status sf_read_body_setup(sf_world *w, float *body12, float *local3);
sf_status sf_read_brick_positions(sf_world *w, float *wpos3);
/* contacts of one scene in the reference's list order (last substep): ids 5 (a, b, bo, ba, bb; scene-local body
 * ids, 0xFFFFFFFF = static, scene-local combined brick ids: static k, body brick n_static + k), f 7 (p 3, n 3,
 * depth), s 8 (jn, jt1, jt2, mn, mt1, mt2, bias, vn0). *n receives the count; buffers may be NULL to query it. */
sf_status sf_read_contacts(sf_world *w, uint32_t scene, uint32_t *ids5, float *f7, float *s8, uint64_t cap,
                           uint64_t *n);
/* manifolds of one scene in (a, b) order: a, b, colour, contact count */
sf_status sf_read_manifolds(sf_world *w, uint32_t scene, uint32_t *out4, uint64_t cap, uint64_t *n);
/* island label per body (world-global id of the island's smallest body; 0xFFFFFFFF = not awake) */
sf_status sf_read_islands(sf_world *w, uint32_t *label);
sf_status sf_read_phi(sf_world *w, float *phi);
/* the solver's f64 potentials (sf_read_phi returns them rounded to f32, the reference's type) */
sf_status sf_read_phi64(sf_world *w, double *phi);
sf_status sf_write_phi(sf_world *w, const float *phi);
sf_status sf_write_ext(sf_world *w, const float *ext);
sf_status sf_read_ext(sf_world *w, float *ext);
/* per static brick: bond 4 (+x, +y, +z, foundation), neighbour 6 (static brick id or 0xFFFFFFFF), material */
sf_status sf_read_bonds(sf_world *w, float *bond4, uint32_t *nb6, uint8_t *mat);
/* joints of the last sf_structure_check, 4 per static brick (+x, +y, +z, foundation): ratio, bond after, and the
 * decision (0 hold, 1 fatigue, 2 fail, 3 crush, 255 absent) with the crushed brick id for crushes */
sf_status sf_read_joints(sf_world *w, float *ratio4, float *bond4, uint8_t *decision4, uint32_t *crushed4);

/* ---- load-path solve without allocation
 * No counterpart in the reference. Some callers cannot allocate GPU memory: a host engine that owns the device and
 * gives this library no allocator of its own, or a frame loop that must not allocate once it is running. For them
 * this entry point solves one structure (every brick given is structure 0, potentials start at 0, as a fresh world's
 * first sf_structure_solve) with no cudaMalloc, no cudaFree and no allocating library call: all of its device
 * scratch is one file-scope array of SF_STATIC_SCRATCH_BYTES (2.7 MB) that every GPU loading the library holds until
 * the process exits. Inputs (lattice cells 3 per brick, material, infill, ext loads or NULL) and outputs (f64
 * potentials per brick, sweeps, final residual) are host buffers of the caller. More than SF_STATIC_MAX_BRICKS
 * bricks, or bricks spread over more than SF_STATIC_MAX_CHUNKS chunks of 8^3 cells, return SF_ERR_CAPACITY.
 * A brick outside the lattice, two bricks in one cell, or a material outside 1..8 return SF_ERR_ARG.
 * The solve stops at tol or at max_sweeps, whichever comes first, and returns SF_OK either way: the caller compares
 * *resid_out with tol. Every brick must reach the ground through bonds (a piece that does not has no finite
 * potential; its potentials grow sweep by sweep and the call returns SF_ERR_VERIFY only once one is non-finite).
 * Each call is synchronous on `stream`: it waits for its own work to finish and reads the results back to the host,
 * so no call can be recorded inside a stream capture. The first call on a device looks up the array's device
 * address (with that device current); the address is kept for the life of the process, so the entry point must not
 * be called again on a device after cudaDeviceReset. Every call reuses the same array: calls whose work overlaps on
 * the GPU race. */
#define SF_STATIC_MAX_BRICKS 8192
#define SF_STATIC_MAX_CHUNKS 128
#define SF_STATIC_SCRATCH_BYTES 2815744
sf_status sf_structure_solve_static(uint32_t n_bricks, const int32_t *xyz, const uint8_t *mat, const uint8_t *infill,
                                    const float *ext, float omega, float tol, uint32_t max_sweeps, double *phi_out,
                                    uint32_t *sweeps_out, double *resid_out, void *stream);

/* ---- narrow phase entry points (batched) */
/* Box-box SAT with face clipping and edge-edge, reduced to 4 points (engine/src/phys.rs:502-628). Boxes are
 * 10 floats: centre 3, quaternion 4, half extents 3. out per pair: count, normal 3, 4 x (point 3, separation). */
sf_status sf_collide_boxes(const float *boxes_a, const float *boxes_b, uint32_t n_pairs, float margin,
                           float *out20, int32_t *count);

/* Convex-cell SAT (gpu/gpu_world.js:421-530 hull_ground / hull_hull, reduce4 :532-554): face axes of both cells,
 * edge-direction crosses, reference-face clipping (up to 16 points, the deepest 8 kept) or edge-edge closest points.
 * hull_data: n_hulls x 80 float4 in the reference's packed layout. Shapes are 11 floats: centre 3, quaternion 4,
 * half extents 3, hull id; a b-shape with a negative hull id is the ground plane. out per pair: normal 3, 0, then
 * 8 x (point 3, separation); reduce != 0 keeps at most 4 points. */
sf_status sf_collide_hulls(const float *hull_data, uint32_t n_hulls, const float *shapes_a, const float *shapes_b,
                           uint32_t n_pairs, float margin, int32_t reduce, float *out36, int32_t *count);

/* ---- the engine crate's box world (engine/src/phys.rs World): oriented boxes, the hashed-grid broadphase, box SAT
 * with face clipping, the soft-step solver (warm start, biased solve, integrate, relax) with anchored patch friction,
 * and island sleep. It replaces World::new + add_box (phys.rs:124-146), World::step (phys.rs:152-243) and the reads
 * of World::bodies / World::stats (phys.rs:108-121); many scenes (independent worlds) step in one launch. */
typedef struct sf_box_world sf_box_world;
typedef struct sf_box_params {       /* Params (engine/src/phys.rs:74-98); defaults phys.rs:99-106 */
    float gravity[3];                /* (0, -9.81, 0) */
    uint32_t substeps;               /* 12 */
    float contact_hertz;             /* 0 = a sixth of the sub-step rate */
    float damping_ratio;             /* 10 */
    float max_push;                  /* 3 m/s */
    float friction;                  /* 0.6 */
    float speculative;               /* 0.02 m */
    float sleep_lin, sleep_ang, sleep_time, sleep_dist, sleep_rot;   /* 0.05, 0.08, 0.5 s, 0.01 m, 0.02 rad */
    int32_t allow_sleep;             /* 1 */
    float cell;                      /* broadphase cell, 1 m */
    float leak;                      /* 1: the soft-step impulse leak as Box2D v3 */
    int32_t anchor;                  /* 1: friction anchors */
    float anchor_push, anchor_slop;  /* 3 m/s, 0 m */
    uint32_t reserved[4];
} sf_box_params;
typedef struct sf_box_stats {        /* Stats (phys.rs:108-110) of the last step, plus the solver's own counts */
    uint32_t awake, pairs, manifolds, points;
    uint32_t colours;                /* colours of the manifold colouring (solve passes per sub-step) */
    uint32_t status;                 /* 0, or capacity flags: 1 grid entries, 2 pairs, 4 manifolds, 8 colours */
    uint32_t rounds;                 /* colouring rounds */
    uint32_t reserved;
    float ms;                        /* device time of the last sf_box_world_step call, all its steps */
    uint64_t steps;                  /* steps taken */
    float phase_ms[5];               /* that call's time in this scene's broadphase, narrow phase and manifolds,
                                      * colouring, sub-steps, write-back and sleep (Stats::t_broad, t_narrow, t_solve) */
    uint32_t reserved2;
} sf_box_stats;
/* boxes: n records of 11 floats (centre 3, quaternion x y z w, half extents 3, density; density 0 = static), scene
 * s = records [scene_first[s], scene_first[s + 1]). Capacities per scene, on average over its boxes: 27 grid entries,
 * 48 broadphase pairs and 8 manifolds a box; and 128 colours. sf_box_world_step returns SF_ERR_CAPACITY past them
 * (that scene's step is left undone; its status flags say which). */
sf_status sf_box_world_create(const float *boxes, const uint32_t *scene_first, uint32_t n_scenes,
                              const sf_box_params *params, sf_box_world **out);
void sf_box_world_destroy(sf_box_world *w);
/* Convex cells in the box world (the WebGPU world's hull shapes, gpu/gpu_world.js:786-833): hull_data holds n_hulls
 * cells of 80 float4 (the packed library, cell 0 the whole cube), hull_ids a cell per box (0 = a plain box). A pair
 * with a cell goes through the convex-cell SAT (a plain box as the whole cube), a cell on the ground through its
 * corners, the first four one patch and the rest a second (manifold b = 0xFFFFFFFE); each reduced to 4 points.
 * The boxes keep their mass and inertia. Call before the first step. */
sf_status sf_box_world_set_hulls(sf_box_world *w, const float *hull_data, uint32_t n_hulls, const uint32_t *hull_ids);
/* nsteps steps of dt for every scene; synchronous. */
sf_status sf_box_world_step(sf_box_world *w, float dt, uint32_t nsteps);
/* 22 floats a box: centre 3, quaternion 4, velocity 3, spin 3, sleep timer, rest pose (centre 3, quaternion 4), awake */
sf_status sf_box_world_read(sf_box_world *w, float *out22);
sf_status sf_box_world_stats(sf_box_world *w, uint32_t scene, sf_box_stats *out);
/* The last step's manifolds of a scene in key order (a, b; the ground as b = 0xFFFFFFFF after a's pairs and a
 * cell's second ground patch), 16 words
 * each: a, b, point count, sticking, normal 3, normal impulses 4, friction impulses 2, twist impulse (f32 bits),
 * colour. *count gets the number of manifolds; at most cap are written. */
sf_status sf_box_world_manifolds(sf_box_world *w, uint32_t scene, uint32_t *out16, uint32_t cap, uint32_t *count);

/* ---- scene pools: the batched and served forms (no counterpart in the reference, which runs one world per wasm
 * instance). A pool is a world of fixed-capacity scene slots; a rigid scene (bodies plus loose static geometry, no
 * load-path structures) is loaded into a slot, stepped with the other slots by sf_world_step / sf_world_step_scenes
 * (slot index = scene index), saved to host memory and restored, bit for bit, into any slot large enough. */
typedef struct sf_pool_slot {
    uint32_t bodies, bricks;    /* body and body-brick capacity */
    uint32_t statics, chunks;   /* static-brick capacity and the 8^3 chunks they may occupy */
} sf_pool_slot;
/* Device bytes a pool of these slots takes (an estimate from the per-element sizes, initial contact capacity of 4
 * per brick included). */
sf_status sf_pool_bytes(uint32_t n_slots, const sf_pool_slot *slots, uint64_t *bytes);
/* A pool has no spare capacity for detached pieces: params with damage or detach_* set return SF_ERR_ARG (contact
 * reduction and warm start are allowed; a slot's warm-start entries start over when it is loaded or cleared). */
sf_status sf_pool_create(uint32_t n_slots, const sf_pool_slot *slots, const sf_params *params, sf_world **out);
/* Load a scene into a slot (replacing what it held); SF_ERR_CAPACITY if it does not fit. */
sf_status sf_pool_load(sf_world *w, uint32_t slot, const sf_scene_desc *scene);
sf_status sf_pool_clear(sf_world *w, uint32_t slot);
/* Host bytes of a snapshot of a scene with these counts, and the snapshot calls: save writes the slot's mutable
 * state (body poses, velocities, rotation caches, sleep state; brick positions and removals) to host memory;
 * restore loads the scene's fixed parts from its description and then that state. */
uint64_t sf_pool_snapshot_bytes(uint32_t n_bodies, uint32_t n_bricks);
sf_status sf_pool_save(sf_world *w, uint32_t slot, void *host, uint64_t cap, uint64_t *bytes);
sf_status sf_pool_restore(sf_world *w, uint32_t slot, const sf_scene_desc *scene, const void *host, uint64_t bytes);
/* The loaded scene's bodies, as sf_read_bodies / sf_write_bodies. */
sf_status sf_pool_read_bodies(sf_world *w, uint32_t slot, float *state13, float *sleep, uint8_t *flags);
sf_status sf_pool_write_bodies(sf_world *w, uint32_t slot, const float *state13, const float *sleep, const uint8_t *flags);

/* ---- serving (no counterpart in the reference): a request loop over resident worlds with continuous batching.
 * Scene-step requests run on a scene pool (one step of every scene with work per tick, in one set of launches;
 * a scene without a slot takes a free one or evicts the least recently used idle scene to pinned host memory);
 * structure-solve requests run on a resident structures world (every structure with work solved in one persistent
 * launch of up to sweeps_per_tick sweeps per tick). The two kinds run on their own threads and streams, so their
 * device work overlaps. With batching = 0 one thread runs the requests one at a time in arrival order, each with
 * its own launches (the plain path). Requests arrive at t_arrival on the server clock (seconds since
 * sf_server_start), so an arrival process can be submitted up front. */
#define SF_REQ_STEP 1
#define SF_REQ_SOLVE 2
typedef struct sf_server sf_server;
typedef struct sf_server_desc {
    uint32_t n_slots;
    const sf_pool_slot *slots;           /* the scene pool (n_slots = 0: no scene requests) */
    const sf_world_desc *structures;     /* the resident structures (NULL: no solve requests) */
    uint64_t budget_bytes;               /* device bytes the resident state may take (0 = no limit): SF_ERR_BUDGET above */
    float dt;                            /* step length of scene requests */
    uint32_t sweeps_per_tick;            /* SOR sweeps per tick of the solve batch (0 = 128) */
    uint32_t batching;                   /* 1 = continuous batching, 0 = one request at a time */
    sf_params params;
} sf_server_desc;
typedef struct sf_request {
    uint32_t kind;                       /* SF_REQ_STEP or SF_REQ_SOLVE */
    uint32_t world;                      /* a scene id from sf_server_add_scene, or a structure id */
    uint32_t nsteps;                     /* STEP */
    float omega, tol;                    /* SOLVE */
    uint32_t max_sweeps;                 /* SOLVE */
    uint32_t n_loads, reserved;          /* SOLVE: ext[load_brick[k]] += load_value[k] before the solve (copied) */
    const uint32_t *load_brick;
    const float *load_value;
    double t_arrival;
    float *out_state13;                  /* STEP, optional: the scene's bodies after the request (13 floats each) */
} sf_request;
typedef struct sf_result {
    uint64_t ticket;
    uint32_t kind, world, status, steps, sweeps, reserved;
    double residual;
    double t_arrival, t_start, t_done;   /* server clock, seconds */
} sf_result;
typedef struct sf_server_stats {
    uint64_t completed, pending, step_ticks, solve_ticks, loads, restores, evictions;
    uint64_t pool_bytes;                 /* device bytes the resident state took at creation */
    double busy_s, now_s;
} sf_server_stats;
sf_status sf_server_create(const sf_server_desc *desc, sf_server **out);
/* Register a scene (deep copy) before sf_server_start; it is loaded into a slot when a request needs it. */
sf_status sf_server_add_scene(sf_server *s, const sf_scene_desc *scene, uint32_t *id);
/* Optional, before sf_server_start: the registered scene's body state (as sf_write_bodies) at its first load, e.g.
 * a world that has already been running (copied). */
sf_status sf_server_set_scene_state(sf_server *s, uint32_t id, const float *state13, const float *sleep,
                                    const uint8_t *flags);
sf_status sf_server_start(sf_server *s);
/* Thread-safe. */
sf_status sf_server_submit(sf_server *s, const sf_request *req, uint64_t *ticket);
/* Finished requests (up to cap), waiting up to wait_ms for the first. */
sf_status sf_server_poll(sf_server *s, sf_result *out, uint32_t cap, uint32_t *n, uint32_t wait_ms);
/* Wait until every submitted request has finished. */
sf_status sf_server_drain(sf_server *s, uint32_t timeout_ms);
sf_status sf_server_get_stats(sf_server *s, sf_server_stats *out);
/* The structures' potentials (FP64), when no request is open. */
sf_status sf_server_read_phi64(sf_server *s, double *phi);
void sf_server_destroy(sf_server *s);

#ifdef __cplusplus
}
#endif
#endif
