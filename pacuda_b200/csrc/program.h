// The host side of a plan: decoding its 64-bit row words, the order-preserving grouping of its
// contribution runs, and the instruction stream the device kernels execute.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#ifdef __CUDACC__
#define PACUDA_HD __host__ __device__ __forceinline__
#else
#define PACUDA_HD inline
#endif

namespace pacuda {

// field widths (W_P .. W_K of pacman_recurrence.h)
enum { WP, WA, WF, WX, WS, WK };

// One decoded row, its operands by name (the row forms of runner/recurrence_runner.cu:10-36 and
// convert/src/program.rs:24-46). An operand a row's op does not have stays 0.
struct Row {
    uint32_t op = 0;       // 1..14
    uint32_t init = 0;     // ops 2-6, 13: the first contribution sets (1) rather than adds
    uint32_t slot = 0;     // ops 2-6: the scale slot; op 12: the mass slot
    uint32_t p0 = 0, p1 = 0;  // ops 2-6, 11, 13: the parent currents
    uint32_t dst = 0;      // ops 2-6, 12, 13: the destination; ops 1, 7-10: the first plane
    uint32_t f0 = 0, f1 = 0;  // ops 2-6, 13: the momentum forms; ops 7-9, 12: f0 is the form
    uint32_t factor = 0;   // the exact factor
    uint32_t count = 0;    // ops 1, 10, 11: the planes or components
    uint32_t amplitude = 0;  // op 11
    uint32_t first = 0;    // op 11: the first component factor
    uint32_t code = 0;     // op 12: the 10-bit wavefunction template
    // op 14: kernel index, input codes, output pairs, direct-capable, and where its codes start
    // in the decoder's binding data (inputs first, then the output components)
    uint32_t kernel = 0, inputs = 0, pairs = 0, direct = 0, data_first = 0;
};

// ops 2-6 (contributions): they form the runs that the grouping below may reorder
PACUDA_HD bool is_contribution(uint32_t op) { return op >= 2 && op <= 6; }

// an instruction of the device stream: 32 bytes
enum InsKind : uint32_t { K_CONTRIB = 1, K_PROP = 2, K_IDENTITY = 3, K_CLEAR = 4, K_CLOSURE = 5, K_SOURCE = 6 };
enum Flag : uint32_t { F_INIT = 1, F_FIRST = 2, F_LAST = 4 };

struct Ins {
    uint32_t head;  // kind | op << 4 | flags << 8 | count << 16
    uint32_t a;     // contribution: parent 0; propagator / identity / clear / source: base; closure: parent 0
    uint32_t b;     // contribution: parent 1; closure: parent 1
    uint32_t c;     // contribution: destination; closure: amplitude plane
    uint32_t f;     // forms: f0 | f1 << 16 (contribution); the form (propagator, source)
    uint32_t s;     // contribution: scale slot; source: mass slot
    uint32_t x;     // exact factor
    uint32_t y;     // closure: first component factor; source: template code
};
static_assert(sizeof(Ins) == 32, "instructions are 32 bytes");

PACUDA_HD uint32_t ins_kind(const Ins &i) { return i.head & 15; }
PACUDA_HD uint32_t ins_op(const Ins &i) { return (i.head >> 4) & 15; }
PACUDA_HD uint32_t ins_flags(const Ins &i) { return (i.head >> 8) & 255; }
PACUDA_HD uint32_t ins_count(const Ins &i) { return i.head >> 16; }

struct Limits {
    uint64_t current_planes, amplitude_planes, forms, scales, factors;
};

// A plan compiled for the device: the instruction stream in the plan's row order (after the
// grouping of contribution runs), the leading source instructions counted apart.
struct Program {
    std::vector<Ins> ins;
    uint32_t sources = 0;     // leading K_SOURCE instructions
    uint32_t flops = 0;       // algorithmic flops per point (fixed per-op counts)
    std::vector<uint32_t> reads_before_write;  // current planes read before any write (live-in)
    std::vector<uint8_t> writes;               // per current plane: written by the program
    Limits need{0, 0, 0, 0, 0};                // the smallest tables the program's references fit
};

// the call's tables hold every reference of the program
inline bool fits(const Program &p, const Limits &l) {
    return p.need.current_planes <= l.current_planes && p.need.amplitude_planes <= l.amplitude_planes &&
           p.need.forms <= l.forms && p.need.scales <= l.scales && p.need.factors <= l.factors;
}

// Status of building a program: 0 ok; otherwise the runner's status code with a message.
struct BuildError {
    int status = 0;
    std::string message;
};

// decode + grouping (when `sort`) + instructions; limits are checked (every plane, form, scale and factor a row
// names lies inside the call's tables)
BuildError build_program(const uint64_t *words, uint32_t count, const uint8_t *width, bool sort,
                         const Limits &limits, Program &out);

// the decoded rows alone (tests and tools)
enum DecodeStatus { DECODE_OK, DECODE_BAD_WORD /* an op outside 1..14, a width above 32 bits */,
                    DECODE_TRUNCATED_BINDING /* an op-14 binding whose codes run past the last word */ };
DecodeStatus decode_rows(const uint64_t *words, uint32_t count, const uint8_t *width, std::vector<Row> &rows,
                         std::vector<uint32_t> &binding_data);
// each maximal run of contribution rows whose destinations are disjoint and which reads none of
// them: its rows gathered per destination, each destination's rows in their order (so every
// destination's sum has the same bits)
void group_contribution_runs(std::vector<Row> &rows);

void contribution_shape(int op, int *c0, int *c1, int *cd);

// an instruction's algorithmic flops (fixed per-op counts)
uint32_t ins_flops(const Ins &i);

}  // namespace pacuda
