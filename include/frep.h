/* frep.h — C-ABI of the B200 F-rep voxelize-and-raytrace library.
 *
 * This is the drop-in boundary for the reference's hot path
 * (MathisBD/f-rep-voxel-rendering, vulkan/): every entry point below names the
 * reference interface it replaces. Plain pointers and sizes only; CUDA streams
 * are passed as `void*` (a cudaStream_t, NULL = the legacy default stream).
 *
 * Conventions
 *   - Every function returns frep_status. The reference has no status codes (it
 *     prints and asserts: vulkan/include/vk_wrapper/vk_check.h:8-18, tape.cpp:
 *     223-227); here each of those failure points returns an error instead.
 *   - Handles are opaque and owned by the library; *_destroy releases them.
 *   - A frep_ctx owns one device's memory arena with an explicit HBM budget.
 *     It is thread-compatible (one host thread at a time), not thread-safe.
 *   - frep_last_error() returns a message for the most recent failure on the
 *     calling thread.
 */
#ifndef FREP_H
#define FREP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum frep_status {
    FREP_OK = 0,
    FREP_ERR_INVALID_ARG = 1,   /* bad pointer, size or enum value                */
    FREP_ERR_OOM = 2,           /* the context's HBM budget or cudaMalloc refused */
    FREP_ERR_CAPACITY = 3,      /* a tree's node or tape pool filled up           */
    FREP_ERR_TIMEOUT = 4,       /* a bounded device loop gave up                  */
    FREP_ERR_CUDA = 5,          /* a CUDA runtime call failed                     */
    FREP_ERR_UNSUPPORTED = 6,   /* valid request outside this build's limits      */
    FREP_ERR_COMPILE = 7        /* the expression could not be compiled to a tape */
} frep_status;

const char* frep_last_error(void);
const char* frep_version(void);

/* ---------------------------------------------------------------------------
 * Expressions and tapes
 * ------------------------------------------------------------------------- */

/* csg::Operator numbering (vulkan/include/csg/expression.h:14-22). */
enum {
    FREP_OP_X = 0, FREP_OP_Y, FREP_OP_Z, FREP_OP_T, FREP_OP_CONST,
    FREP_OP_SIN, FREP_OP_COS, FREP_OP_EXP, FREP_OP_NEG, FREP_OP_SQRT,
    FREP_OP_ADD, FREP_OP_SUB, FREP_OP_MUL, FREP_OP_DIV, FREP_OP_MIN, FREP_OP_MAX
};

/* Tape opcodes (vulkan/include/csg/tape.h:15-30). */
enum {
    FREP_TAPE_CONST = 0, FREP_TAPE_SIN, FREP_TAPE_COS, FREP_TAPE_ADD, FREP_TAPE_SUB,
    FREP_TAPE_MUL, FREP_TAPE_DIV, FREP_TAPE_MIN, FREP_TAPE_MAX, FREP_TAPE_EXP,
    FREP_TAPE_NEG, FREP_TAPE_SQRT, FREP_TAPE_COPY
};

/* A flattened csg::Expr DAG: node i = (ops[i], in0[i], in1[i], consts[i]);
 * inputs refer to earlier nodes; unused inputs are ignored. This is how a
 * csg::Expr (shared_ptr DAG, expression.h:29-100) crosses the boundary. */
typedef struct frep_dag {
    uint32_t n_nodes;
    const uint8_t* ops;
    const uint32_t* in0;
    const uint32_t* in1;
    const float* consts;
    uint32_t root;
} frep_dag;

typedef struct frep_tape frep_tape;

typedef struct frep_tape_info {
    uint32_t n_instr;         /* csg::Tape::instructions.size()                 */
    uint32_t n_slots;         /* csg::Tape::GetSlotCount()                      */
    uint32_t n_consts;        /* csg::Tape::constantPool.size()                 */
    uint32_t n_minmax;        /* MIN/MAX instructions (pruning choice points)   */
    uint32_t fits_reference;  /* 1 if the 8-bit reference encoding can hold it  */
    uint32_t uses_time;       /* 1 if slot 3 (T) is read                        */
} frep_tape_info;

/* Replaces csg::Tape::Tape(Expr) (vulkan/src/csg/tape.cpp:14-228): simplify,
 * topologically sort, pool constants, allocate slots. Same instruction stream
 * as the reference for every tape its 8-bit encoding can hold; wide encoding
 * so that large scenes compile. */
frep_status frep_tape_compile(const frep_dag* dag, frep_tape** out);

/* Compiler options. const_reload_distance applies to tapes beyond the 8-bit
 * encoding only (whose instruction stream is this library's own): a use of a
 * pooled constant more than this many instructions after its last load gets
 * a CONST of its own and slots are allocated again, so that shared constants
 * do not hold slots across the tape (the 256-primitive scene: 23 -> 14
 * slots for 15 % more instructions; each slot costs every resident warp a
 * shared-memory row on the device). 0 = default (8), 0xFFFFFFFF = never. */
typedef struct frep_tape_opts {
    uint32_t const_reload_distance;
    uint32_t reserved[3];
} frep_tape_opts;
frep_status frep_tape_compile_opts(const frep_dag* dag, const frep_tape_opts* opts, frep_tape** out);

/* Accepts a tape in the reference's own upload format
 * (vulkan/src/engine/voxelizer.cpp:385-398: op | out<<8 | inA<<16 | inB<<24)
 * with its constant pool. */
frep_status frep_tape_from_reference(const uint32_t* instrs, uint32_t n_instr, const float* consts,
                                     uint32_t n_consts, frep_tape** out);

/* Accepts a tape in this library's wide encoding (frep_tape_get_instrs), e.g.
 * one saved earlier or edited (new constants, same structure). No
 * counterpart in the reference. */
frep_status frep_tape_from_wide(const uint64_t* instrs, uint32_t n_instr, frep_tape** out);

frep_status frep_tape_get_info(const frep_tape* tape, frep_tape_info* info);

/* Wide instruction words (8 bytes each): op bits 0-7, out 16-31, inA 32-47,
 * inB 48-63; for CONST bits 32-63 hold the float. cap = capacity of `out`. */
frep_status frep_tape_get_instrs(const frep_tape* tape, uint64_t* out, uint32_t cap);

/* csg::Tape::instructions / constantPool in the reference's 8-bit encoding;
 * FREP_ERR_UNSUPPORTED when the tape does not fit it (fits_reference == 0). */
frep_status frep_tape_get_reference(const frep_tape* tape, uint32_t* instrs, float* consts);

/* Replaces csg::Tape::Eval (tape.cpp:274-302) on the host: n points, 4 floats
 * (x, y, z, t) each. */
frep_status frep_tape_eval(const frep_tape* tape, const float* xyzt, uint32_t n, float* out);

void frep_tape_destroy(frep_tape* tape);

typedef struct frep_ctx frep_ctx;

/* csg::Tape::Eval (tape.cpp:274-302) on the device for many points at once:
 * n points of (x, y, z, t) in host memory, n values back in host memory. The
 * operations and rounding of the last-level point pass (point.comp:2-63), so
 * a value here is the one that pass compares with 0. Synchronous; working
 * memory comes from the context's budget for the duration of the call. */
frep_status frep_tape_eval_device(frep_ctx* ctx, const frep_tape* tape, const float* xyzt, uint32_t n, float* out);

/* The interval extension the level passes compute (tape_eval_interval,
 * interval.comp:8-160) over n caller-given boxes: box i is 6 floats (low x,
 * y, z, high x, y, z) in host memory, T = [tape_time, tape_time]; out[2i],
 * out[2i+1] = the interval's low and high bound. rounding: FREP_ROUND_*
 * (below). With FREP_ROUND_OUTWARD every interval contains the tape's exact
 * value at every point of its box. Synchronous. */
frep_status frep_tape_eval_intervals(frep_ctx* ctx, const frep_tape* tape, const float* boxes, uint32_t n,
                                     float tape_time, uint32_t rounding, float* out);

/* ---------------------------------------------------------------------------
 * Device context
 * ------------------------------------------------------------------------- */

/* Opens `device` with an HBM budget in bytes (0 = 90% of free memory). Replaces
 * the Vulkan device/VMA set-up of EngineBase::Init (engine_base.cpp:45-160). */
frep_status frep_ctx_create(int device, uint64_t hbm_budget_bytes, frep_ctx** out);
void frep_ctx_destroy(frep_ctx* ctx);
/* Bytes of the budget currently held by trees and scratch. */
frep_status frep_ctx_memory(const frep_ctx* ctx, uint64_t* used, uint64_t* budget);

/* ---------------------------------------------------------------------------
 * Voxelization (sparse tree build)
 * ------------------------------------------------------------------------- */

#define FREP_MAX_LEVELS 8

/* VoxelStorage's inputs (vulkan/include/engine/voxel_storage.h:15-22):
 * gridDims (children per axis per level; each a multiple of 4, 4..32),
 * lowVertex and worldSize. */
typedef struct frep_grid {
    uint32_t levels;
    uint32_t dims[FREP_MAX_LEVELS];
    float low_vertex[3];
    float world_size;
} frep_grid;

enum {
    FREP_ROUND_NEAREST = 0,   /* the reference's round-to-nearest intervals       */
    FREP_ROUND_OUTWARD = 1,   /* directed rounding: every interval is conservative */
    FREP_ROUND_HYBRID = 2     /* outward intervals intersected with affine forms  */
};
/* FREP_ROUND_HYBRID is this library's own mode, the working counterpart of
 * the reference's abandoned affine evaluator (vulkan/shaders/tape/affine.comp,
 * commented out): every slot also carries an affine form over the cell's
 * axes, c + x ex + y ey + z ez + [-e, e], with every rounding error added to e
 * (rounded up), and keeps its outward interval intersected with the form's
 * range. Conservative like FREP_ROUND_OUTWARD and never looser; much tighter
 * where intervals suffer from the dependency problem (polynomials such as
 * the reference's TangleCube, x^4 - 8 x^2 + ...), so fewer cells stay
 * ambiguous. The interval passes run one cell per lane with 32-byte slot rows. */

typedef struct frep_voxelize_opts {
    uint32_t rounding;        /* FREP_ROUND_*                                        */
    uint32_t shorten;         /* 1 = prune min/max into shortened child tapes (ref.) */
    uint64_t node_words;      /* node pool capacity in u32 words (0 = automatic)     */
    uint64_t tape_words;      /* tape pool capacity in u64 words (0 = automatic)     */
    uint32_t point_cells_per_lane; /* last-level pass: cells per lane, 2, 4 or 8 (0 =
                                    * automatic: 4 when dim^3/32 is a multiple of 4);
                                    * it must divide dim^3/32; batches and the server
                                    * take 2 or 4 only */
    uint32_t separate_tapes;  /* 0: cells of a 32-cell group whose shortened tapes
                               * are identical share one copy (~3x less tape pool);
                               * 1: one copy per cell, as the reference stores them */
} frep_voxelize_opts;

typedef struct frep_tree frep_tree;

/* Creates an empty tree for `grid` with its own node and tape pools (carved
 * from the context's budget). The tree can be re-voxelized many times. */
frep_status frep_tree_create(frep_ctx* ctx, const frep_grid* grid, const frep_voxelize_opts* opts,
                             frep_tree** out);
void frep_tree_destroy(frep_tree* tree);

/* Replaces Voxelizer::Voxelize(waitSem, tapeTime) (vulkan/src/engine/
 * voxelizer.cpp:429-440, with VoxelizeLevel :295-329). Builds the whole tree
 * level by level on `stream` WITHOUT a host round trip per level; returns when
 * the work is enqueued. Overflow of the pools is reported by frep_tree_sync. */
frep_status frep_voxelize(frep_ctx* ctx, frep_tree* tree, const frep_tape* tape, float tape_time,
                          void* stream);

/* Animated scenes: the same voxelization as frep_voxelize (the same nodes,
 * masks and tape contents), built faster by copying from `prev` (the previous
 * frame's tree) every subtree whose node tape never reads the time input and
 * is identical to prev's node tape at the same level and coordinates; only the
 * time-dependent part is evaluated again. Replaces the reference's full
 * re-voxelization per frame (Application::Draw, application.cpp:68-79).
 *   - prev: another tree of the same context, same grid, rounding and
 *     shortening, voxelized before (any tape and time; a subtree is copied only
 *     when its tape matches exactly). Its voxelization must be ordered before
 *     this call's work (the same stream, or synchronized), and prev must not be
 *     voxelized again until this call's work is done. A prev whose pools
 *     overflowed is not used (everything is evaluated).
 *   - Typical use: two trees A and B alternate, frame k voxelizes into one
 *     with the other as prev.
 *   - The first call allocates two side arrays of node_words / 8 + 1 u32 for
 *     the tree (per node, where it was copied from; per level, the nodes to
 *     evaluate).
 *   - frep_tree_work and frep_tree_fp32_ops count only the evaluated nodes.
 * FREP_ERR_INVALID_ARG: prev null, equal to tree, not voxelized, or with
 * another grid / options. */
frep_status frep_voxelize_reuse(frep_ctx* ctx, frep_tree* tree, const frep_tree* prev, const frep_tape* tape,
                                float tape_time, void* stream);

/* Same voxelization as frep_voxelize, for callers that cannot allocate device
 * memory when they voxelize (a fixed budget reserved up front, a frame loop
 * that must not hit cudaMalloc's implicit synchronisation, or an application
 * whose allocator owns every buffer). It makes no allocation: the interval
 * pass's per-warp scratch is an 8 MiB array in the library's device image
 * instead of a cudaMalloc'd buffer, and the root tape is copied straight from
 * `tape` (pageable memory: the call returns once the driver has staged it).
 * No counterpart in the reference.
 *   - Limit: each warp of a block needs k * (n + 2m) 32-bit words (n
 *     instructions, m of them MIN/MAX, each term rounded up to 32; k = 1 or 2
 *     cells per lane, as the plan for the tape's slot count picks), and one
 *     block (1 or 4 warps) must fit the 8 MiB, 2^21 words. Every root tape
 *     with n + 2m <= 262,000 is accepted whatever the plan; longer ones only
 *     when the plan uses fewer cells per lane or warps per block, and
 *     FREP_ERR_UNSUPPORTED otherwise (the tree is untouched and stays usable).
 *     Long tapes run on fewer blocks than frep_voxelize uses, so they take
 *     longer.
 *   - Its first call on a device looks up the array's device address; make that
 *     first call before any stream capture.
 *   - Every call on a device shares the one array: calls whose work overlaps
 *     on the GPU (different streams, no ordering between them) race. Nothing
 *     in it needs to start at zero; each call overwrites what it reads.
 * The tree, its pools and the tape must still be created by the caller. */
frep_status frep_voxelize_static_scratch(frep_ctx* ctx, frep_tree* tree, const frep_tape* tape,
                                         float tape_time, void* stream);

/* Waits for the tree's stream and reads its header. Replaces the per-level
 * childCount readback (voxelizer.cpp:326-328) and PrintStats (:442-478). */
typedef struct frep_tree_info {
    uint32_t levels;
    uint32_t dims[FREP_MAX_LEVELS];
    uint32_t node_count[FREP_MAX_LEVELS];      /* interiorNodeCount              */
    uint64_t node_offset[FREP_MAX_LEVELS];     /* in u32 words                   */
    uint32_t node_size[FREP_MAX_LEVELS];       /* in u32 words                   */
    uint64_t tape_size_sum[FREP_MAX_LEVELS];   /* stats_buf.tape_size_sum        */
    uint32_t tape_size_max[FREP_MAX_LEVELS];   /* stats_buf.max_tape_size        */
    uint64_t node_words_used, node_words_cap;
    uint64_t tape_words_used, tape_words_cap;
    uint32_t overflow;                          /* bit 0 node pool, bit 1 tapes   */
    uint32_t root_tape_words;
} frep_tree_info;
frep_status frep_tree_sync(frep_tree* tree, frep_tree_info* info);

/* Copies the device buffers to the host (for export and parity checks). The
 * node layout is the reference's (node.comp:1-72, voxel_storage.h:57-88):
 * per level contiguous; node = [tapeIdx, cx, cy, cz, leafMask[dim^3/32],
 * interiorMask[dim^3/32], childList[dim^3]], last level = [tapeIdx, cx, cy, cz,
 * leafMask, unused]. tapeIdx indexes the tape pool in u64 words; a tape is
 * [header: n_instr (u32) | reserved (u32)] followed by n_instr wide words. */
frep_status frep_tree_copy_nodes(frep_tree* tree, uint32_t* dst, uint64_t n_words);

/* Profiling: when enabled, frep_voxelize records a CUDA event pair around each
 * level pass on its stream; frep_tree_timings waits for them and returns the
 * device time of every level pass of the last voxelization, in milliseconds. */
frep_status frep_tree_set_profiling(frep_tree* tree, int enable);
frep_status frep_tree_timings(frep_tree* tree, float ms[FREP_MAX_LEVELS]);
/* Cell-instructions evaluated per level by the last voxelization: the number
 * of (cell, tape instruction) pairs the interval and point passes executed. */
frep_status frep_tree_work(frep_tree* tree, uint64_t cell_instr[FREP_MAX_LEVELS]);
/* Op-weighted FP32 work per level of the last voxelization: for every
 * (cell, instruction) pair, the number of FP32 operations of the reference's
 * interval formula for that opcode (interval levels) or 1 per arithmetic
 * instruction (the last, point level). The roofline numerator. */
frep_status frep_tree_fp32_ops(frep_tree* tree, uint64_t ops[FREP_MAX_LEVELS]);
frep_status frep_tree_copy_tapes(frep_tree* tree, uint64_t* dst, uint64_t n_words);

/* ---------------------------------------------------------------------------
 * Rendering
 * ------------------------------------------------------------------------- */

enum { FREP_PERSPECTIVE = 0, FREP_ORTHOGRAPHIC = 1 };

/* Camera (vulkan/include/engine/camera.h:6-41). forward/up need not be
 * normalised or orthogonal: right = normalize(forward x up), up' = right x forward
 * (camera.cpp:16-27). Perspective uses the horizontal fov_deg
 * (raytracer.cpp:177-181); orthographic uses ortho_width world units across. */
typedef struct frep_camera {
    float position[3];
    float forward[3];
    float up[3];
    float fov_deg;
    float ortho_width;
    uint32_t projection;
    uint32_t width, height;
    uint32_t jitter;          /* 0 = ray through pixel corner (parity), 1 = jittered */
    float jitter_seed;        /* the reference seeds rand() with the wall clock      */
} frep_camera;

#define FREP_MAX_LIGHTS 8
/* Directional lights and background (raytracer.cpp:183-192). Directions are
 * the direction the light travels; the library normalises them. shadow_mask
 * bit i = cast a shadow ray toward light i (the reference's shadow ray is
 * commented out at raytracer/main.comp:125-133). */
typedef struct frep_lights {
    uint32_t count;
    float direction[FREP_MAX_LIGHTS][3];
    float color[FREP_MAX_LIGHTS][4];
    float ambient[4];
    float background[4];
    uint32_t shadow_mask;
} frep_lights;

/* Fills `lights` with the reference's two hard-coded lights, 0.2 ambient and a
 * black background, no shadows. */
frep_status frep_lights_default(frep_lights* lights);

/* Output buffers (device pointers; any may be NULL):
 *   rgba8 : width*height*4 bytes, row-major, the reference's rgba8 image layer
 *   hits  : width*height frep_hit records (for parity and debugging) */
typedef struct frep_hit {
    float t;                  /* ray parameter of the hit (Hit.t)               */
    float normal[3];          /* normalised gradient at the hit point           */
    uint32_t level;           /* tree level of the hit cell, 0xFFFFFFFF = miss  */
    uint32_t node;            /* node id at that level                          */
    uint32_t cell;            /* bit index z + dim*y + dim^2*x inside the node  */
    uint32_t steps;           /* DDA iterations spent                           */
} frep_hit;

typedef struct frep_image {
    uint8_t* rgba8;
    frep_hit* hits;
} frep_image;

/* Replaces Raytracer::Trace(waitSem, camera, tapeTime) (vulkan/src/engine/
 * raytracer.cpp:243-272 and raytracer/main.comp:161-183). Enqueued on `stream`. */
frep_status frep_render(frep_ctx* ctx, const frep_tree* tree, const frep_camera* camera,
                        const frep_lights* lights, float tape_time, const frep_image* out,
                        void* stream);

/* Temporal multi-sample resolve (renderer/triangle.frag:14-23 with
 * render_target.cpp:36-56 and raytracer.cpp:163-164): the reference renders
 * one jittered frame per display frame into layer (frame % count) of an
 * image array and the fragment shader averages the layers. Here:
 *   frep_resolve_layers — out = mean of n_layers consecutive rgba8 images
 *     (device memory, width*height*4 bytes each): rgb rounded to nearest
 *     (ties up) from the exact sum, alpha 255;
 *   frep_render_temporal — renders n_samples jittered frames of the tree into
 *     `layers` (device, n_samples*width*height*4 bytes; sample i uses jitter
 *     seed camera->jitter_seed + i) and resolves them into rgba8. */
frep_status frep_resolve_layers(const uint8_t* layers, uint32_t n_layers, uint32_t width, uint32_t height,
                                uint8_t* out, void* stream);
frep_status frep_render_temporal(frep_ctx* ctx, const frep_tree* tree, const frep_camera* camera,
                                 const frep_lights* lights, float tape_time, uint32_t n_samples, uint8_t* layers,
                                 uint8_t* rgba8, void* stream);

/* ---------------------------------------------------------------------------
 * Compact trees (render-ready, export / import)
 *
 * Replaces SceneBuilder's compaction and layout (vulkan/src/engine/
 * scene_builder.cpp: BuildNode :91-156, LayoutNode :199-238; the layout notes
 * of vulkan/README.md:22-54): the voxelizer's tree is not compactified
 * (nodes can be empty or have only leaf cells), and every interior node
 * carries a full dim^3 child list. A compact tree
 *   - numbers the nodes of every level in depth-first preorder, children in
 *     ascending cell order (LayoutNode), so the children of a node are
 *     consecutive and are found from one base index and a popcount: a
 *     non-last node is [tapeIdx, leafMask[W], interiorMask[W], prefix[W],
 *     base] (W = dim^3/32; prefix[w] = interior cells in words before w; the
 *     child of interior cell i is base + prefix[i/32] + the interior cells
 *     before i in its word), a last-level node [tapeIdx, leafMask[W]];
 *   - keeps one copy of every tape its nodes use (tapeIdx: u64 word index
 *     into the compact tree's own tape pool, records as in frep_tree);
 *   - with FREP_COMPACT_PRUNE, also applies BuildNode's rules bottom-up: a
 *     child node with no leaf and no interior cell is dropped, one whose
 *     cells are all leaves becomes a leaf cell of its parent. The solid
 *     voxels are the same; rays that hit a collapsed node hit its parent's
 *     cell instead (same depth t, normal from the parent's tape). The root is
 *     always kept. FREP_COMPACT_LAYOUT keeps every node and mask: renders
 *     give the same hits (cells, depths, normals) as the source tree.
 * ------------------------------------------------------------------------- */

enum { FREP_COMPACT_LAYOUT = 0, FREP_COMPACT_PRUNE = 1 };

typedef struct frep_compact frep_compact;

typedef struct frep_compact_info {
    uint32_t levels;
    uint32_t dims[FREP_MAX_LEVELS];
    uint32_t mode;                              /* FREP_COMPACT_*                       */
    uint32_t n_slots;                           /* slots of the longest tape (render)   */
    uint32_t node_count[FREP_MAX_LEVELS];
    uint64_t node_offset[FREP_MAX_LEVELS];      /* u32 words                            */
    uint32_t node_size[FREP_MAX_LEVELS];        /* u32 words                            */
    uint64_t node_words;                        /* u32 words of the node pool           */
    uint64_t tape_words;                        /* u64 words of the tape pool           */
    uint64_t device_bytes;                      /* held on the device                   */
} frep_compact_info;

/* Builds the compact form of a voxelized tree (which is left unchanged and
 * may then be destroyed or voxelized again). Blocking: waits for the tree's
 * voxelization, runs the compaction on `stream` and waits for it. Device
 * memory: the result (charged to the context's budget) plus, while the call
 * runs, working buffers of the result's upper bound (when pruning, copied
 * into an exact one at the end), 16 bytes per node of the largest level,
 * 1 byte per node (pruning) and 1/2 byte per tape word.
 * FREP_ERR_CAPACITY: the tree's pools overflowed; FREP_ERR_INVALID_ARG: not
 * voxelized or a bad mode. */
frep_status frep_tree_compact(frep_ctx* ctx, frep_tree* tree, uint32_t mode, void* stream, frep_compact** out);
frep_status frep_compact_get_info(const frep_compact* compact, frep_compact_info* info);
/* Waits for the device (renders of the tree may be in flight on any stream),
 * then frees it. */
void frep_compact_destroy(frep_compact* compact);

/* Raytracer::Trace over a compact tree: the same camera, lights, shading and
 * outputs as frep_render; frep_hit.node is the node's preorder index. */
frep_status frep_render_compact(frep_ctx* ctx, const frep_compact* compact, const frep_camera* camera,
                                const frep_lights* lights, float tape_time, const frep_image* out, void* stream);

/* Serialised compact tree ("blob"): a frep_compact_header, then the node pool
 * (node_words u32), then the tape pool (tape_words u64); each section starts
 * on an 8-byte boundary (the node section is zero-padded to one). Little
 * endian, position independent: it can be written to a file and imported in
 * another process or on another device. */
typedef struct frep_compact_header {
    char magic[8];                              /* "FREPCT01"                           */
    uint32_t version;                           /* 1                                    */
    uint32_t levels;
    uint32_t dims[FREP_MAX_LEVELS];
    float low_vertex[3];
    float world_size;
    uint32_t mode;
    uint32_t n_slots;
    uint32_t node_count[FREP_MAX_LEVELS];
    uint64_t node_words;
    uint64_t tape_words;
} frep_compact_header;

/* Writes the blob of `compact` to host memory. *size = its size in bytes;
 * dst = NULL asks for the size only; a dst smaller than it (cap) is
 * FREP_ERR_INVALID_ARG. Blocking. */
frep_status frep_compact_export(const frep_compact* compact, void* dst, uint64_t cap, uint64_t* size);

/* Checks a blob on the host (no device needed): header fields, section sizes,
 * every node's masks, prefix counts and child ranges (each child referenced
 * once, in preorder), every tape index and record, and every instruction's
 * opcode and slots against n_slots. FREP_OK or FREP_ERR_INVALID_ARG with the
 * first problem in frep_last_error(). */
frep_status frep_compact_check(const void* blob, uint64_t size);

/* Uploads a blob (checked first with frep_compact_check) into a new compact
 * tree of `ctx`. Blocking. */
frep_status frep_compact_import(frep_ctx* ctx, const void* blob, uint64_t size, frep_compact** out);

/* ---------------------------------------------------------------------------
 * Batching: many scenes per launch
 * ------------------------------------------------------------------------- */

/* A fixed set of trees that are voxelized and rendered together. Every level
 * pass is ONE launch over all the trees (warps take work items from any tree
 * through one device cursor), and all frames are one launch. No counterpart in
 * the reference, which voxelizes one scene at a time with a host fence per
 * level (voxelizer.cpp:295-329). All trees must use the same rounding. */
typedef struct frep_batch frep_batch;

frep_status frep_batch_create(frep_ctx* ctx, frep_tree* const* trees, uint32_t n, frep_batch** out);
void frep_batch_destroy(frep_batch* batch);

/* Voxelizes tree i from tapes[i] at tape_times[i] (tape_times may be NULL:
 * all 0). Enqueued on `stream`; frep_tree_sync works per tree afterwards. */
frep_status frep_batch_voxelize(frep_batch* batch, const frep_tape* const* tapes, const float* tape_times,
                                void* stream);

/* Replaces the batch's tree set (any size, same rounding); plans, scratch
 * and upload areas are kept and grown as needed. */
frep_status frep_batch_set_trees(frep_batch* batch, frep_tree* const* trees, uint32_t n);

/* Renders frame i of tree frame_trees[i] (any voxelized trees of the batch's
 * context, repeats allowed) with cameras[i] into images[i]: one launch. */
frep_status frep_batch_render_frames(frep_batch* batch, const frep_tree* const* frame_trees, uint32_t n_frames,
                                     const frep_camera* cameras, const frep_lights* lights,
                                     const float* tape_times, const frep_image* images, void* stream);

/* Renders tree i with cameras[i] into images[i] (one launch for all frames). */
frep_status frep_batch_render(frep_batch* batch, const frep_camera* cameras, const frep_lights* lights,
                              const float* tape_times, const frep_image* images, void* stream);

/* Voxelize + render. With use_graph != 0 the whole sequence (one upload, the
 * level passes, the frames) is captured into a CUDA graph on first use and
 * replayed while the batch keeps its shape (same tape lengths, frame sizes and
 * buffers); a new shape is captured again. */
frep_status frep_batch_run(frep_batch* batch, const frep_tape* const* tapes, const float* tape_times,
                           const frep_camera* cameras, const frep_lights* lights, const frep_image* images,
                           int use_graph, void* stream);

typedef struct frep_batch_info {
    uint32_t n_trees;
    uint32_t voxelize_launches;        /* kernels one voxelization of the batch launches */
    uint64_t upload_bytes;             /* host->device bytes of its last voxelization   */
    uint64_t device_bytes;             /* the batch's own scratch + upload area          */
    uint32_t interval_warps_per_block; /* the plan in use (0 before the first run)       */
    uint32_t point_warps_per_block;
    /* cells per lane of the root level's pass for the current tree set: 2 when
     * its root cells fill the grid, else 1 (0 before the first run) */
    uint32_t root_cells_per_lane;
} frep_batch_info;
frep_status frep_batch_get_info(const frep_batch* batch, frep_batch_info* info);

/* Tapes per block of the level passes: each warp of a block runs its own
 * work items (and so its own tape); 0 = chosen from the shared memory a warp
 * needs (4 when four warps fit in 200 KB, else 1), 1 or 4 = that many where
 * shared memory allows. Takes effect at the next voxelization. */
frep_status frep_batch_set_tuning(frep_batch* batch, uint32_t interval_warps_per_block,
                                  uint32_t point_warps_per_block);

/* ---------------------------------------------------------------------------
 * Pool sizing and the batch autotuner. The reference fixes one scene's
 * branching by hand (gridDims, vulkan/src/main.cpp:16) and sizes its buffers
 * for the worst case (voxel_storage.h:45-47, 512 MiB of tapes); a batch of
 * hundreds of scenes needs both chosen per scene.
 * ------------------------------------------------------------------------- */

/* Node and tape words each (tape, grid) needs: one voxelization (outward
 * rounding, shortening on) into a scratch tree per distinct grid, grown by
 * doubling on overflow, then the words used times (1 + margin) plus 4096.
 * tape_times may be NULL (all 0). Blocking. */
frep_status frep_fit_pools(frep_ctx* ctx, const frep_tape* const* tapes, const frep_grid* grids,
                           const float* tape_times, uint32_t n, float margin, uint64_t* node_words,
                           uint64_t* tape_words);

/* Tuned choices: per class of scenes (effective resolution per axis, tape
 * size class: < 256, < 1024, < 4096 or more instructions) a grid branching and
 * the last level's cells per lane, and for the whole batch the tapes per block
 * of the level passes. */
typedef struct frep_tuning frep_tuning;
frep_status frep_tuning_create(frep_tuning** out);
void frep_tuning_destroy(frep_tuning* tuning);
/* JSON keyed by device name; load takes `device`'s entry, else "NVIDIA B200",
 * else the file's first. save keeps the other devices' entries. */
frep_status frep_tuning_load(frep_tuning* tuning, const char* path, const char* device);
frep_status frep_tuning_save(const frep_tuning* tuning, const char* path, const char* device);
/* The choice for a scene: *levels = 0 when its class has none. */
frep_status frep_tuning_lookup(const frep_tuning* tuning, uint32_t resolution, uint32_t n_instr, uint32_t* levels,
                               uint32_t dims[FREP_MAX_LEVELS], uint32_t* point_cells_per_lane);
/* The tapes per block to pass to frep_batch_set_tuning (0 = automatic). */
frep_status frep_tuning_warps(const frep_tuning* tuning, uint32_t* interval_warps_per_block,
                              uint32_t* point_warps_per_block);

typedef struct frep_autotune_opts {
    uint32_t per_class;      /* scenes timed per class (0 = 4)                             */
    uint32_t reps;           /* timed runs per candidate; the median counts (0 = 5)        */
    uint32_t width, height;  /* frame size of the timed renders (0 = 512 x 512)            */
    float margin;            /* a candidate replaces the incumbent only when faster by this
                              * fraction (0 = 0.03)                                        */
    uint32_t force;          /* 1: tune every class afresh, cached choices ignored         */
    uint32_t refine;         /* 1: re-time cached classes too, the cached choice first      */
} frep_autotune_opts;

/* Fills `tuning` for every class present among the n scenes (tapes[i] at
 * effective resolution resolutions[i], one of 64, 128, 256, 512, 1024,
 * rendered with cameras[i] and `lights`, grid from low_vertex / world_size):
 * each candidate branching and last-level tile is timed as batched voxelize +
 * render of up to per_class scenes of the class under CUDA graph replay (the
 * median of reps runs); then the tapes per block on up to 32 scenes spread
 * over the batch. The incumbent of a class (its cached choice, else the
 * first candidate) is kept unless a candidate beats it by `margin`, so a
 * repeated tuning keeps its choices. Classes already in `tuning` are skipped
 * unless force or refine. Blocking; allocates and frees its own trees. */
frep_status frep_batch_autotune(frep_ctx* ctx, const frep_tape* const* tapes, const uint32_t* resolutions,
                                const frep_camera* cameras, uint32_t n, const frep_lights* lights,
                                const float low_vertex[3], float world_size, const frep_autotune_opts* opts,
                                frep_tuning* tuning);

/* Profiling of plain (non-graph) batch calls: with profiling on,
 * frep_batch_voxelize and frep_batch_render record events between their
 * launches. frep_batch_timings waits for them and returns device milliseconds:
 * ms[3 l + k] = level l's pass of kind k (0 interval, 1 point with 4 cells per
 * lane, 2 point with 2 cells per lane; each with its work-scan launch),
 * ms[3 FREP_MAX_LEVELS] = root copy + header reset, ms[3 FREP_MAX_LEVELS + 1]
 * = the frames (0 if none were rendered since profiling was enabled). */
frep_status frep_batch_set_profiling(frep_batch* batch, int enable);
frep_status frep_batch_timings(frep_batch* batch, float ms[3 * FREP_MAX_LEVELS + 2]);

/* ---------------------------------------------------------------------------
 * Serving (no counterpart in the reference, whose Application voxelizes and
 * renders one scene per frame, application.cpp:60-93)
 *
 * A request loop with continuous batching: requests (a registered scene, a
 * camera, a tape time, a host image) are queued by frep_server_submit from
 * any thread; a scheduler thread forms a step from whatever is queued (up to
 * max_batch requests) whenever fewer than max_inflight steps are on the
 * device, so requests that arrive while others run join the next step and
 * the device works through steps back to back. A step voxelizes, in one
 * batched launch per level pass, the scenes that are not resident at the
 * requested time and renders every request of the step in one launch; the
 * images are copied to the requests' host buffers in the same stream.
 * Trees (nodes + shortened tapes) stay resident in one device arena of
 * hbm_budget bytes; a request for a resident scene at the same tape time
 * (any time, for scenes that do not read T) is a re-render only. A scene
 * that does not fit is admitted after evicting least recently used trees; a
 * request that cannot be admitted waits. Pools are sized from
 * frep_voxelize_opts when given, else estimated and then refitted from the
 * scene's measured use; a voxelization that overflows its pools is retried
 * with doubled pools (at most 4 times, then FREP_ERR_CAPACITY).
 * Diagnostics: with the environment variable FREP_SERVER_SLOW_MS set to a
 * number of milliseconds when the server is created, every step whose host
 * enqueue takes at least that long prints one line to stderr with the time
 * of each phase (tree headers, voxelization: plans and scratch, upload area,
 * staging and launches; frame area, render, read-backs).
 * ------------------------------------------------------------------------- */

typedef struct frep_server frep_server;

typedef struct frep_server_config {
    uint64_t hbm_budget;      /* bytes of the tree arena (0 = 80 % of the context's free budget) */
    uint32_t max_batch;       /* requests per step (0 = 512)                                     */
    uint32_t max_inflight;    /* steps enqueued on the device at once (0 = 2)                    */
    uint32_t interval_warps_per_block, point_warps_per_block;  /* frep_batch_set_tuning         */
} frep_server_config;

typedef struct frep_request {
    uint64_t scene;           /* from frep_server_add_scene                                      */
    frep_camera camera;       /* width x height of the image                                     */
    float tape_time;
    uint8_t* rgba8;           /* host buffer of width*height*4 bytes, written by the device copy;
                                 page-locked memory lets the copy run asynchronously             */
} frep_request;

enum { FREP_REQ_QUEUED = 0, FREP_REQ_RUNNING = 1, FREP_REQ_DONE = 2, FREP_REQ_FAILED = 3 };

typedef struct frep_request_status {
    int32_t state;            /* FREP_REQ_*                                                      */
    int32_t status;           /* frep_status of a failed request                                 */
    uint32_t voxelized;       /* 1: this request's step voxelized the scene; 0: re-render only   */
    uint32_t retries;
    double latency_ms;        /* submit -> image in the host buffer (done requests)              */
} frep_request_status;

typedef struct frep_server_stats {
    uint64_t submitted, completed, failed, voxelized, rerendered, evictions, steps;
    uint64_t resident_trees, resident_bytes, arena_bytes;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* latency of requests completed since the last reset */
    double scenes_per_s;      /* completed / (last completion - first submit), since the reset  */
    /* Since the last reset: the longest time the scheduler held the server's
     * lock to form one step (submits wait for it), the longest host time to
     * enqueue one step, and the most trees evicted while forming one step. */
    double max_plan_ms, max_enqueue_ms;
    uint64_t max_step_evictions;
} frep_server_stats;

/* lights: used for every request (NULL = frep_lights_default). */
frep_status frep_server_create(frep_ctx* ctx, const frep_server_config* config, const frep_lights* lights,
                               frep_server** out);
/* Finishes the work on the device, stops the threads, frees everything. */
void frep_server_destroy(frep_server* server);
/* Registers a scene (the tape is copied). opts: rounding, shortening, pool
 * sizes (0 = estimated), last-level cells per lane. */
frep_status frep_server_add_scene(frep_server* server, const frep_tape* tape, const frep_grid* grid,
                                  const frep_voxelize_opts* opts, uint64_t* scene);
frep_status frep_server_submit(frep_server* server, const frep_request* request, uint64_t* request_id);
frep_status frep_server_poll(frep_server* server, uint64_t request_id, frep_request_status* status);
/* Waits until the request is done or failed, at most timeout_ms
 * (FREP_ERR_TIMEOUT). */
frep_status frep_server_wait(frep_server* server, uint64_t request_id, uint32_t timeout_ms,
                             frep_request_status* status);
/* Forgets a finished request (its status can no longer be polled). A
 * long-running caller releases every request it has waited for. */
frep_status frep_server_release(frep_server* server, uint64_t request_id);
/* Waits until every submitted request is done or failed. */
frep_status frep_server_drain(frep_server* server, uint32_t timeout_ms);
/* Statistics; reset != 0 clears the latency record and throughput window. */
frep_status frep_server_get_stats(frep_server* server, int reset, frep_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* FREP_H */
