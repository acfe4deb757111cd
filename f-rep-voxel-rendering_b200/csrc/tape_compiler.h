// Tape compiler: expression DAG -> linear, register-allocated tape.
//
// Produces the same instruction sequence, slot assignment and constant pool as
// the reference's csg::Tape (vulkan/src/csg/tape.cpp:14-228), but
//   * in a wide encoding (16-bit slots, the constant stored inline), so that
//     tapes with more than 256 slots or constants compile, and
//   * with hash-consing and memoised structural comparison, so that tapes of
//     tens of thousands of instructions compile in milliseconds.
// When a tape fits the reference's 8-bit encoding, ref_instrs/const_pool hold it
// byte-for-byte as csg::Tape::instructions / constantPool.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace frep {

// csg::Operator numbering (vulkan/include/csg/expression.h:14-22).
enum class ExprOp : uint8_t {
    X = 0, Y, Z, T, CONST, SIN, COS, EXP, NEG, SQRT, ADD, SUB, MUL, DIV, MIN, MAX
};

// Tape opcodes (vulkan/include/csg/tape.h:15-30, vulkan/shaders/tape/tape.comp:15-27).
enum TapeOp : uint32_t {
    OP_CONST = 0, OP_SIN = 1, OP_COS = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5, OP_DIV = 6,
    OP_MIN = 7, OP_MAX = 8, OP_EXP = 9, OP_NEG = 10, OP_SQRT = 11, OP_COPY = 12, OP_COUNT = 13
};

// Wide instruction word (8 bytes):
//   bits  0..7   opcode
//   bits 16..31  output slot
//   bits 32..47  input slot A       (CONST: bits 32..63 = the float constant)
//   bits 48..63  input slot B
inline uint64_t encode_instr(uint32_t op, uint32_t out, uint32_t a, uint32_t b) {
    return (uint64_t)op | ((uint64_t)out << 16) | ((uint64_t)a << 32) | ((uint64_t)b << 48);
}
inline uint64_t encode_const(uint32_t out, float c) {
    uint32_t bits;
    static_assert(sizeof(bits) == sizeof(c), "float must be 32-bit");
    __builtin_memcpy(&bits, &c, 4);
    return (uint64_t)OP_CONST | ((uint64_t)out << 16) | ((uint64_t)bits << 32);
}
inline uint32_t instr_op(uint64_t w) { return (uint32_t)(w & 0xFF); }
inline uint32_t instr_out(uint64_t w) { return (uint32_t)((w >> 16) & 0xFFFF); }
inline uint32_t instr_a(uint64_t w) { return (uint32_t)((w >> 32) & 0xFFFF); }
inline uint32_t instr_b(uint64_t w) { return (uint32_t)((w >> 48) & 0xFFFF); }
inline float instr_const(uint64_t w) {
    uint32_t bits = (uint32_t)(w >> 32);
    float c;
    __builtin_memcpy(&c, &bits, 4);
    return c;
}

struct DagNode {
    uint8_t op;
    uint32_t in0, in1;
    float constant;
};

struct CompiledTape {
    std::vector<uint64_t> instrs;      // wide encoding
    uint32_t n_slots = 0;              // csg::Tape::GetSlotCount()
    uint32_t n_minmax = 0;             // MIN/MAX instruction count
    bool uses_time = false;            // slot 3 (T) is read
    // Reference encoding, valid when fits_reference: op | out<<8 | inA<<16 | inB<<24.
    bool fits_reference = false;
    std::vector<uint32_t> ref_instrs;
    std::vector<float> const_pool;     // csg::Tape::constantPool order
};

// Returns an empty string on success, else a message. The DAG must be
// topologically ordered (inputs before users) with root < n.
// const_reload: for tapes beyond the reference's 8-bit encoding, a use that
// lies more than this many instructions after its constant's last load gets a
// CONST of its own (slots reallocated); 0 = never.
std::string compile_tape(const DagNode* nodes, uint32_t n, uint32_t root, CompiledTape* out,
                         uint32_t const_reload = 8);

// Imports a tape in the wide encoding (as frep_tape_get_instrs returns it):
// validates the opcodes and derives the slot count, MIN/MAX count and whether
// T is read.
std::string import_wide_tape(const uint64_t* instrs, uint32_t n, CompiledTape* out);

// Imports a tape in the reference's 8-bit encoding with its constant pool.
std::string import_reference_tape(const uint32_t* instrs, uint32_t n, const float* consts,
                                  uint32_t n_consts, CompiledTape* out);

// Host point interpreter over a wide tape (the semantics of csg::Tape::Eval,
// tape.cpp:274-302, with the library's own sin/cos/exp).
float eval_point_host(const std::vector<uint64_t>& instrs, uint32_t n_slots, float x, float y,
                      float z, float t);

}  // namespace frep
