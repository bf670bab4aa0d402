// Coding tables of the EBCOT tier-1 coder and the MQ arithmetic coder.
//
// These are data of the coding format and must match the reference value for value (each table
// is defined once, as a macro, and instantiated as device constant memory (c_*) and as a host
// array (h_*) for the host build of the tier-1 kernel bodies):
//  - MQ probability-state machine, 94 states = 47 probability states x 2 MPS senses
//    (mq.c:197-291), packed here as  p | mps << 16 | next_if_mps << 17 | next_if_lps << 24;
//  - significance-context maps for low-pass, high-pass and doubly-high-pass subbands indexed
//    by 15*h + 5*v + d neighbour counts (tier1.c:231-262);
//  - sign-context reduction SIG2XI and the sign context/flip table XI2CONT (tier1.c:264-275);
//  - log2 fraction table used by slope2log (tier1.c:200-216).
// The distortion tables of tier1.c:139-165 are linear and are evaluated in closed form
// (see dist_ts / dist_tm), the run-length table (tier1.c:181-184) by a leading-zero count.
#pragma once
#include <cstdint>

namespace bwcb {
namespace dev {

// context labels (mq.h:68-73)
constexpr int kCtxSig = 0, kCtxRun = 9, kCtxSign = 10, kCtxMag = 15, kCtxUni = 18, kCtxTotal = 19;

#define BWCB_MQ_STATES \
    { \
    0x30025601u, 0x06043401u, 0x09061801u, 0x0C080AC1u, 0x1D0A0521u, 0x214C0221u, \
    0x350E5601u, 0x0E105401u, 0x0E124801u, 0x0E143801u, 0x11163001u, 0x12182401u, \
    0x141A1C01u, 0x153A1601u, 0x3D1E5601u, 0x0E205401u, 0x0F225101u, 0x10244801u, \
    0x11263801u, 0x12283401u, 0x132A3001u, 0x132C2801u, 0x142E2401u, 0x15302201u, \
    0x16321C01u, 0x17341801u, 0x18361601u, 0x19381401u, 0x1A3A1201u, 0x1B3C1101u, \
    0x1C3E0AC1u, 0x1D4009C1u, 0x1E4208A1u, 0x1F440521u, 0x20460441u, 0x214802A1u, \
    0x224A0221u, 0x234C0141u, 0x244E0111u, 0x25500085u, 0x26520049u, 0x27540025u, \
    0x28560015u, 0x29580009u, 0x2A5A0005u, 0x2B5A0001u, 0x2E5C5601u, 0x01615601u, \
    0x35633401u, 0x38651801u, 0x3B670AC1u, 0x4C690521u, 0x50AB0221u, 0x066D5601u, \
    0x3D6F5401u, 0x3D714801u, 0x3D733801u, 0x40753001u, 0x41772401u, 0x43791C01u, \
    0x44991601u, 0x0E7D5601u, 0x3D7F5401u, 0x3E815101u, 0x3F834801u, 0x40853801u, \
    0x41873401u, 0x42893001u, 0x428B2801u, 0x438D2401u, 0x448F2201u, 0x45911C01u, \
    0x46931801u, 0x47951601u, 0x48971401u, 0x49991201u, 0x4A9B1101u, 0x4B9D0AC1u, \
    0x4C9F09C1u, 0x4DA108A1u, 0x4EA30521u, 0x4FA50441u, 0x50A702A1u, 0x51A90221u, \
    0x52AB0141u, 0x53AD0111u, 0x54AF0085u, 0x55B10049u, 0x56B30025u, 0x57B50015u, \
    0x58B70009u, 0x59B90005u, 0x5AB90001u, 0x5DBB5601u, \
    }
__constant__ uint32_t c_mq_states[94] = BWCB_MQ_STATES;
static const uint32_t h_mq_states[94] = BWCB_MQ_STATES;

// initial state of each context: significance -> 4, run -> 3, uniform -> 46, others -> 0
// (mq.c:368-375)
__host__ __device__ __forceinline__ uint8_t mq_initial_state(int ctx) {
  return ctx == kCtxSig ? 4 : ctx == kCtxRun ? 3 : ctx == kCtxUni ? 46 : 0;
}

// significance contexts (offsets from kCtxSig) for the three subband classes
#define BWCB_SIG2CTX \
    { \
    {0, 1, 2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 5, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, \
    8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8}, \
    {0, 1, 2, 2, 2, 5, 6, 6, 6, 6, 8, 8, 8, 8, 8, 3, 3, 3, 3, 3, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, \
    4, 4, 4, 4, 4, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8}, \
    {0, 3, 6, 8, 8, 1, 4, 7, 8, 8, 2, 5, 7, 8, 8, 1, 4, 7, 8, 8, 2, 5, 7, 8, 8, 2, 5, 7, 8, 8, \
    2, 5, 7, 8, 8, 2, 5, 7, 8, 8, 2, 5, 7, 8, 8}}
__constant__ uint8_t c_sig2ctx[3][45] = BWCB_SIG2CTX;
static const uint8_t h_sig2ctx[3][45] = BWCB_SIG2CTX;

// neighbour pair (significance bits 0/1, sign bits 2/3) -> 0 negative, 1 none, 2 positive
#define BWCB_SIG2XI \
    {1, 2, 2, 2, 1, 0, 2, 1, 1, 2, 0, 1, 1, 0, 0, 0}
__constant__ uint8_t c_sig2xi[16] = BWCB_SIG2XI;
static const uint8_t h_sig2xi[16] = BWCB_SIG2XI;

// (horizontal << 2 | vertical) -> sign context | flip << 7
#define BWCB_XI2CONT \
    { \
    (uint8_t)(kCtxSign + 4) | 0x80, (uint8_t)(kCtxSign + 3) | 0x80, (uint8_t)(kCtxSign + 2) | 0x80, \
    0, \
    (uint8_t)(kCtxSign + 1) | 0x80, (uint8_t)(kCtxSign + 0),        (uint8_t)(kCtxSign + 1), \
    0, \
    (uint8_t)(kCtxSign + 2),        (uint8_t)(kCtxSign + 3),        (uint8_t)(kCtxSign + 4)}
__constant__ uint8_t c_xi2cont[11] = BWCB_XI2CONT;
static const uint8_t h_xi2cont[11] = BWCB_XI2CONT;

#define BWCB_FRAC2LOG \
    { \
    0,   1,   2,   4,   5,   7,   8,   9,   11,  12,  14,  15,  16,  18,  19,  21,  22,  23, \
    25,  26,  27,  29,  30,  31,  33,  34,  35,  37,  38,  39,  40,  42,  43,  44,  46,  47, \
    48,  49,  51,  52,  53,  54,  56,  57,  58,  59,  61,  62,  63,  64,  65,  67,  68,  69, \
    70,  71,  73,  74,  75,  76,  77,  78,  80,  81,  82,  83,  84,  85,  87,  88,  89,  90, \
    91,  92,  93,  94,  96,  97,  98,  99,  100, 101, 102, 103, 104, 105, 106, 108, 109, 110, \
    111, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 122, 123, 124, 125, 126, 127, 128, \
    129, 131, 132, 133, 134, 135, 136, 137, 138, 139, 140, 140, 141, 142, 143, 144, 145, 146, \
    147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 162, 163, \
    164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 173, 174, 175, 176, 177, 178, 179, 180, \
    181, 181, 182, 183, 184, 185, 186, 187, 188, 188, 189, 190, 191, 192, 193, 194, 194, 195, \
    196, 197, 198, 199, 200, 200, 201, 202, 203, 204, 205, 205, 206, 207, 208, 209, 209, 210, \
    211, 212, 213, 214, 214, 215, 216, 217, 218, 218, 219, 220, 221, 222, 222, 223, 224, 225, \
    225, 226, 227, 228, 229, 229, 230, 231, 232, 232, 233, 234, 235, 235, 236, 237, 238, 239, \
    239, 240, 241, 242, 242, 243, 244, 245, 245, 246, 247, 247, 248, 249, 250, 250, 251, 252, \
    253, 253, 254, 255}
__constant__ uint16_t c_frac2log[256] = BWCB_FRAC2LOG;
static const uint16_t h_frac2log[256] = BWCB_FRAC2LOG;

// distortion decrease of a newly significant sample, indexed by the 5 magnitude bits below the
// current bit plane (tier1.c:157-165: 49152 + 6144 i)
__host__ __device__ __forceinline__ int32_t dist_ts(uint32_t i) { return 49152 + 6144 * (int32_t)i; }

// distortion change of a refined sample, indexed by the 6 magnitude bits below the current
// plane (tier1.c:139-155: a V-shaped table with its minimum -16384 at index 32)
__host__ __device__ __forceinline__ int32_t dist_tm(uint32_t i) {
  return (i < 32) ? 49152 - 2048 * (int32_t)i : 2048 * (int32_t)i - 81920;
}

}  // namespace dev
}  // namespace bwcb
