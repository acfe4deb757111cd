// CPU oracle for the F-rep voxelize + raytrace path — TEST INFRASTRUCTURE.
//
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// arm may load it. It is the checker, never part of the product path.
//
// It restates, in plain C++, the reference's GPU semantics, each function citing
// the shader it follows (paths relative to the reference repository):
//   interval evaluation  vulkan/shaders/tape/interval.comp:8-160
//   tape shortening      vulkan/shaders/tape/shorten.comp:10-223
//   level pass / tree    vulkan/shaders/voxelizer/main.comp:19-170, node.comp,
//                        vulkan/src/engine/voxelizer.cpp:200-251, :429-440
//   point evaluation     vulkan/shaders/tape/point.comp:2-63
//   gradient             vulkan/shaders/tape/gradient.comp:4-88
//   raytracer            vulkan/shaders/raytracer/main.comp:24-183,
//                        vulkan/src/engine/raytracer.cpp:157-212, camera.cpp:16-27
// Parity pin: the reference's own tests hold no golden vectors for this path,
// and its GLSL cannot run here (no graphics stack), so the shader restatement
// is "parity unpinned" against the reference's GPU output. What IS pinned:
// the tape compiler against the reference's csg::Tape (byte-exact,
// tests/test_compiler.py), the point interpreter against csg::Tape::Eval
// (bit-exact for algebraic tapes), outward intervals of sampled cells of
// whole trees against FP64 dense sampling with a rigorous error bound
// (tests/test_containment.py; the device's in tests/test_gpu_containment.py),
// and oracle_directed against exact rational arithmetic
// (tests/test_math_ulp.py).
//
// Every float operation rounds on its own (built with -ffp-contract=off);
// transcendentals come from include/frep/frep_math.h, the library's definition.
#pragma once
#include <cstdint>

extern "C" {

// ---- single-tape primitives (for unit tests) --------------------------------
// tape: wide instruction words (include/frep.h), n_slots from the compiler.
// rounding: 0 = round-to-nearest (reference), 1 = outward.
// choices (optional, n_minmax bytes): 1 FIRST, 2 SECOND, 3 BOTH per MIN/MAX.
void oracle_eval_interval(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                          const float* lo3, const float* hi3, float t, int rounding,
                          float* out_lohi, uint8_t* choices);
// Every instruction's result interval (trace: 2 floats per instruction;
// rounding 0 or 1), for tests of properties of the intermediate values.
void oracle_eval_interval_trace(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                                const float* lo3, const float* hi3, float t, int rounding,
                                float* trace);
float oracle_eval_point(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots, float x,
                        float y, float z, float t);
void oracle_eval_gradient(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots, float x,
                          float y, float z, float t, float* out_grad3);
// Shortens a tape given the choices of one interval evaluation. Returns the
// output length; writes the shortened tape to out (capacity n_instr) only if
// it is shorter, else returns n_instr and leaves out untouched.
uint32_t oracle_shorten(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                        const uint8_t* choices, uint32_t n_minmax, uint64_t* out);

// Directed-rounding helpers, exposed so tests can check them against exact
// rational arithmetic. op: 0 add, 1 sub, 2 mul, 3 div, 4 sqrt(a); dir: -1 down, +1 up.
float oracle_directed(int op, int dir, float a, float b);

// ---- whole tree -------------------------------------------------------------
// Builds the sparse tree exactly as the level passes do. Returns a handle.
void* oracle_voxelize(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                      const uint32_t* dims, uint32_t levels, const float* low_vertex,
                      float world_size, float tape_time, int rounding, int shorten,
                      int threads);
void oracle_tree_free(void* tree);
// info: [levels, node_count[8], node_size[8] (u32 words), node_offset[8] (u32
// words), total_node_words, total_tape_words]  -> 1 + 8*3 + 2 = 27 uint64 values.
void oracle_tree_info(void* tree, uint64_t* info);
void oracle_tree_nodes(void* tree, uint32_t* dst);
void oracle_tree_tapes(void* tree, uint64_t* dst);
// Work counters: per level, cell-instructions evaluated (interval or point).
void oracle_tree_work(void* tree, uint64_t* cell_instr8);

// Compaction of a voxelized tree (vulkan/src/engine/scene_builder.cpp): a new
// tree handle in the same node layout whose levels are numbered in depth-first
// preorder (LayoutNode, :199-238: children in ascending cell order). prune != 0
// also applies BuildNode's rules (:91-156) bottom-up: a child node with no leaf
// or interior cell is dropped, one whose cells are all leaves becomes a leaf
// cell of its parent. The root is always kept. Tapes are unchanged (same pool).
void* oracle_compact(void* tree, int prune);

// ---- rendering --------------------------------------------------------------
// camera: [pos3, fwd3, up3, fov_deg, ortho_width, projection, width, height,
// jitter, jitter_seed] as floats (width/height/projection/jitter as values).
// lights: count, dir[8][3], color[8][4], ambient[4], background[4], shadow_mask.
// hits: width*height records of 8 x 32-bit (t, n.xyz, level, node, cell, steps).
void oracle_render(void* tree, const float* camera, uint32_t n_lights, const float* light_dir,
                   const float* light_color, const float* ambient, const float* background,
                   uint32_t shadow_mask, float tape_time, uint8_t* rgba8, uint32_t* hits,
                   int threads);
}
