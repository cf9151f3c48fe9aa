// The host side of a plan: decoding its 64-bit row words, the order-preserving sort of its
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

// one decoded row (reference: runner/recurrence_runner.cu:913-975; convert/src/program.rs:60-114)
struct Row {
    int op;          // 1..14
    uint32_t f[8];   // fields in word order
    uint32_t data_first = 0, data_count = 0;  // op 14: its codes in Plan::binding_data
};

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

// A plan compiled for the device: the instruction stream in the reference's row order (after
// the sort), the leading source instructions counted apart.
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

// decode + sort + instructions; limits are checked (every plane, form, scale and factor a row
// names lies inside the call's tables)
BuildError build_program(const uint64_t *words, uint32_t count, const uint8_t *width, bool sort,
                         const Limits &limits, Program &out);

// the decoded rows alone (tests and tools)
bool decode_rows(const uint64_t *words, uint32_t count, const uint8_t *width, std::vector<Row> &rows,
                 std::vector<uint32_t> &binding_data);
void sort_contribution_runs(std::vector<Row> &rows);

void contribution_shape(int op, int *c0, int *c1, int *cd);

// an instruction's algorithmic flops (fixed per-op counts)
uint32_t ins_flops(const Ins &i);

}  // namespace pacuda
