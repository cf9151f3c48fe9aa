// Host compilation of a plan's words into the device instruction stream.
//
// The row words follow the format of runner/recurrence_runner.cu:10-36 and
// convert/src/program.rs:24-114 (`convert/CONVENTIONS.md` names the operands): a 4-bit op in the
// low bits, then the op's operands from the least significant bit up, each as wide as the call's
// `width` entry for its kind (or 1 or 10 bits); op 14 is followed by data words of two 32-bit
// codes each. Here the layouts are a table of (operand, width) per op and a word is read at bit
// offsets, so a field that would start past bit 63 reads 0, as shifting the word does.
//
// Contribution runs: a run whose destinations are disjoint and which reads none of them may run
// its rows in any order that keeps each destination's own order (the reference sorts such runs
// by destination, recurrence_runner.cu:977-1007). Here each destination's rows are gathered at
// the place of its first row, so a destination's sum becomes one run of rows (F_FIRST .. F_LAST,
// its sum kept in registers) with the same operations in the same order.
#include "program.h"

#include <algorithm>
#include <unordered_map>

namespace pacuda {

void contribution_shape(int op, int *c0, int *c1, int *cd) {
    // (parent 0 components, parent 1 components, written components): CONVENTIONS.md's vertex types
    static const int shape[5][3] = {{2, 4, 2}, {2, 4, 2}, {6, 4, 4}, {4, 4, 6}, {4, 4, 4}};
    const int *s = shape[op - 2];
    *c0 = s[0];
    *c1 = s[1];
    *cd = s[2];
}

namespace {

// the width of a field: an index into the call's `width` table, or a fixed width
enum FieldWidth : uint8_t { ONE_BIT = 6, TEN_BITS = 7 };

struct Field {
    uint32_t Row::*operand;
    uint8_t width;
};

struct Layout {
    uint8_t fields;
    Field field[8];
};

// the operands of each op, least significant first (ops 1 .. 13; 14 is read apart)
const Layout &layout_of(uint32_t op) {
    static const Layout contribution{8, {{&Row::init, ONE_BIT}, {&Row::slot, WS}, {&Row::p0, WP}, {&Row::p1, WP},
                                         {&Row::dst, WP}, {&Row::f0, WF}, {&Row::f1, WF}, {&Row::factor, WX}}};
    static const Layout clear{2, {{&Row::dst, WP}, {&Row::count, WP}}};
    static const Layout propagator{3, {{&Row::dst, WP}, {&Row::f0, WF}, {&Row::factor, WX}}};
    static const Layout identity{3, {{&Row::dst, WP}, {&Row::count, WK}, {&Row::factor, WX}}};
    static const Layout closure{6, {{&Row::p0, WP}, {&Row::p1, WP}, {&Row::amplitude, WA}, {&Row::factor, WX},
                                    {&Row::first, WX}, {&Row::count, WK}}};
    static const Layout source{5, {{&Row::dst, WP}, {&Row::f0, WF}, {&Row::factor, WX}, {&Row::slot, WS},
                                   {&Row::code, TEN_BITS}}};
    static const Layout symjit{7, {{&Row::init, ONE_BIT}, {&Row::p0, WP}, {&Row::p1, WP}, {&Row::dst, WP},
                                   {&Row::f0, WF}, {&Row::f1, WF}, {&Row::factor, WX}}};
    switch (op) {
    case 1: return clear;
    case 7: case 8: case 9: return propagator;
    case 10: return identity;
    case 11: return closure;
    case 12: return source;
    case 13: return symjit;
    default: return contribution;
    }
}

// `n` (at most 32) bits of `word` from bit `at`; bits past the word's end are 0
uint32_t bits_at(uint64_t word, unsigned at, unsigned n) {
    if (n == 0 || at >= 64) return 0;
    return (uint32_t)((word >> at) & ((1ull << n) - 1));
}

// the component interval [lo, hi) a row touches
struct Span {
    uint32_t lo, hi;
};

bool meets(const std::vector<Span> &sorted, Span s) {
    // the first interval that ends after s starts; s meets it if it starts before s ends
    auto it = std::upper_bound(sorted.begin(), sorted.end(), s.lo, [](uint32_t v, const Span &x) { return v < x.hi; });
    return it != sorted.end() && it->lo < s.hi;
}

// whether the contribution rows [begin, end) may be regrouped (see group_contribution_runs)
bool regroupable(const std::vector<Row> &rows, size_t begin, size_t end) {
    std::vector<Span> dest;  // one interval per destination, as wide as its widest row
    for (size_t k = begin; k < end; k++) {
        int c0, c1, cd;
        contribution_shape((int)rows[k].op, &c0, &c1, &cd);
        dest.push_back({rows[k].dst, rows[k].dst + (uint32_t)cd});
    }
    std::sort(dest.begin(), dest.end(), [](const Span &x, const Span &y) { return x.lo != y.lo ? x.lo < y.lo : x.hi > y.hi; });
    std::vector<Span> merged;  // equal starts merged into the widest
    for (const Span &s : dest)
        if (merged.empty() || merged.back().lo != s.lo) merged.push_back(s);
    for (size_t k = 1; k < merged.size(); k++)
        if (merged[k].lo < merged[k - 1].hi) return false;  // two destinations share components
    for (size_t k = begin; k < end; k++) {
        int c0, c1, cd;
        contribution_shape((int)rows[k].op, &c0, &c1, &cd);
        if (meets(merged, {rows[k].p0, rows[k].p0 + (uint32_t)c0}) || meets(merged, {rows[k].p1, rows[k].p1 + (uint32_t)c1}))
            return false;  // the run reads what it writes
    }
    return true;
}

}  // namespace

DecodeStatus decode_rows(const uint64_t *words, uint32_t count, const uint8_t *width, std::vector<Row> &rows,
                         std::vector<uint32_t> &binding_data) {
    rows.clear();
    binding_data.clear();
    uint8_t w[8];
    for (int k = 0; k < 6; k++) {
        if (width[k] > 32) return DECODE_BAD_WORD;
        w[k] = width[k];
    }
    w[ONE_BIT] = 1;
    w[TEN_BITS] = 10;
    uint32_t n = 0;
    while (n < count) {
        const uint64_t word = words[n++];
        Row r;
        r.op = (uint32_t)(word & 15);
        if (r.op == 0 || r.op == 15) return DECODE_BAD_WORD;
        if (r.op == 14) {
            // kernel (16 bits from bit 4), inputs (8 from 20), output pairs (8 from 28), direct (1 from 36)
            r.kernel = bits_at(word, 4, 16);
            r.inputs = bits_at(word, 20, 8);
            r.pairs = bits_at(word, 28, 8);
            r.direct = bits_at(word, 36, 1);
            r.data_first = (uint32_t)binding_data.size();
            const uint32_t codes = r.inputs + r.pairs, data_words = (codes + 1) / 2;
            if (data_words > count - n) return DECODE_TRUNCATED_BINDING;
            for (uint32_t k = 0; k < codes; k++) binding_data.push_back(bits_at(words[n + k / 2], 32 * (k & 1), 32));
            n += data_words;
            rows.push_back(r);
            continue;
        }
        const Layout &l = layout_of(r.op);
        unsigned at = 4;
        for (unsigned k = 0; k < l.fields; k++) {
            const unsigned width_k = w[l.field[k].width];
            r.*(l.field[k].operand) = bits_at(word, at, width_k);
            at += width_k;
        }
        rows.push_back(r);
    }
    return DECODE_OK;
}

void group_contribution_runs(std::vector<Row> &rows) {
    std::vector<uint32_t> rank;
    std::vector<Row> grouped;
    size_t begin = 0;
    while (begin < rows.size()) {
        if (!is_contribution(rows[begin].op)) {
            begin++;
            continue;
        }
        size_t end = begin;
        while (end < rows.size() && is_contribution(rows[end].op)) end++;
        if (end - begin > 1 && regroupable(rows, begin, end)) {
            // rank = the order of each destination's first row; a stable counting sort by rank
            std::unordered_map<uint32_t, uint32_t> rank_of;  // destination -> rank
            rank.assign(end - begin, 0);
            for (size_t k = begin; k < end; k++)
                rank[k - begin] = rank_of.emplace(rows[k].dst, (uint32_t)rank_of.size()).first->second;
            std::vector<uint32_t> start(rank_of.size() + 1, 0);
            for (uint32_t x : rank) start[x + 1]++;
            for (size_t g = 1; g < start.size(); g++) start[g] += start[g - 1];
            grouped.resize(end - begin);
            for (size_t k = begin; k < end; k++) grouped[start[rank[k - begin]]++] = rows[k];
            std::copy(grouped.begin(), grouped.end(), rows.begin() + begin);
        }
        begin = end;
    }
}

namespace {

Ins make(uint32_t kind, uint32_t op, uint32_t flags, uint32_t count) {
    Ins i{};
    i.head = kind | op << 4 | flags << 8 | count << 16;
    return i;
}

bool within(uint64_t first, uint64_t n, uint64_t limit) { return first <= limit && n <= limit - first; }

// algorithmic flops per row: a complex product 6, a complex sum 2, a real-complex product 2,
// a division or square root 1 (counted from the arithmetic of arith.cuh)
uint32_t row_flops(const Ins &i) {
    switch (ins_kind(i)) {
    case K_CONTRIB:
        switch (ins_op(i)) {
        case 2: case 3: return 2 * (4 * 6 + 3 * 2) + 6 + 2 * 8;        // 8 products, 6 sums; scale; 2 x (mul + add)
        case 4: return 4 * (3 * 6 + 2 * 2) + 6 + 4 * 8;
        case 5: return 6 * (2 * 6 + 2) + 6 + 6 * 8;
        default: return (4 * 6 + 3 * 2) + 2 * (4 * 2 + 3 * 2) + 4 * (1 + 2 + 2 * 6 + 2 + 2 + 2) + 6 + 4 * 8;
        }
    case K_PROP:
        if (ins_op(i) == 9) return 7 + 1 + 6 + 2 + 4 * 6;
        return 7 + 1 + 2 + 2 * (4 * 2 + 3 * 2) + 2 * 6;
    case K_IDENTITY: return 6 * i.b;
    case K_CLOSURE: return 20 * i.s;
    case K_SOURCE: return 30;
    default: return 0;
    }
}

}  // namespace

uint32_t ins_flops(const Ins &i) { return row_flops(i); }

BuildError build_program(const uint64_t *words, uint32_t count, const uint8_t *width, bool sort,
                         const Limits &lim, Program &out) {
    BuildError err;
    std::vector<Row> rows;
    std::vector<uint32_t> binding_data;
    switch (decode_rows(words, count, width, rows, binding_data)) {
    case DECODE_OK: break;
    case DECODE_TRUNCATED_BINDING:  // a symjit binding: refused as the rows below
        err.status = 3;
        err.message = "a symjit binding whose codes run past the last word";
        return err;
    default:
        err.status = 2;
        err.message = "a word with an op outside 1..14 or a field width above 32 bits";
        return err;
    }
    for (const Row &r : rows)
        if (r.op == 13 || r.op == 14) {
            // as a runner built without generated symjit kernels (recurrence_runner.cu:1141-1145)
            err.status = 3;
            err.message = "a symjit row, but this runner has no symjit kernels";
            return err;
        }
    if (sort) group_contribution_runs(rows);
    out.ins.clear();
    out.ins.reserve(rows.size());
    out.flops = 0;
    uint64_t P = lim.current_planes;
    auto same_destination = [&](size_t k, uint32_t dst) {
        return k < rows.size() && is_contribution(rows[k].op) && rows[k].dst == dst;
    };
    for (size_t n = 0; n < rows.size(); n++) {
        const Row &r = rows[n];
        Ins i{};
        bool ok = true;
        if (is_contribution(r.op)) {
            const bool first = n == 0 || !same_destination(n - 1, r.dst), last = !same_destination(n + 1, r.dst);
            i = make(K_CONTRIB, r.op, (r.init ? F_INIT : 0) | (first ? F_FIRST : 0) | (last ? F_LAST : 0), 0);
            i.s = r.slot; i.a = r.p0; i.b = r.p1; i.c = r.dst; i.x = r.factor;
            // the forms are read by op 6 only (a form index must fit 16 bits here)
            i.f = r.op == 6 ? ((r.f0 & 0xffff) | (r.f1 << 16)) : 0;
            int c0, c1, cd;
            contribution_shape((int)r.op, &c0, &c1, &cd);
            ok = within(r.p0, c0, P) && within(r.p1, c1, P) && within(r.dst, cd, P) && r.slot < lim.scales &&
                 r.factor < lim.factors &&
                 (r.op != 6 || (r.f0 < lim.forms && r.f1 < lim.forms && r.f0 < 65536 && r.f1 < 65536));
        } else if (r.op == 1) {
            i = make(K_CLEAR, 1, 0, 0);
            i.a = r.dst; i.b = r.count;
            ok = within(r.dst, r.count, P);
        } else if (r.op >= 7 && r.op <= 9) {
            i = make(K_PROP, r.op, 0, 0);
            i.a = r.dst; i.f = r.f0; i.x = r.factor;
            ok = within(r.dst, r.op == 9 ? 4 : 2, P) && r.f0 < lim.forms && r.factor < lim.factors;
        } else if (r.op == 10) {
            i = make(K_IDENTITY, 10, 0, 0);
            i.a = r.dst; i.b = r.count; i.x = r.factor;
            ok = within(r.dst, r.count, P) && r.factor < lim.factors;
        } else if (r.op == 11) {
            i = make(K_CLOSURE, 11, 0, 0);
            i.a = r.p0; i.b = r.p1; i.c = r.amplitude; i.x = r.factor; i.y = r.first;
            i.s = r.count;  // the component count
            ok = within(r.p0, r.count, P) && within(r.p1, r.count, P) && r.amplitude < lim.amplitude_planes &&
                 r.factor < lim.factors && within(r.first, r.count, lim.factors);
        } else {  // 12
            i = make(K_SOURCE, 12, 0, 0);
            i.a = r.dst; i.f = r.f0; i.x = r.factor; i.s = r.slot; i.y = r.code;
            int comps = (r.code & 7) == 0 ? 1 : (r.code & 7) == 1 ? 2 : 4;
            ok = within(r.dst, comps, P) && r.f0 < lim.forms && r.factor < lim.factors && r.slot < lim.scales;
        }
        if (!ok) {
            err.status = 2;
            err.message = "row " + std::to_string(n) + " (op " + std::to_string(r.op) +
                          ") names a plane, form, scale or factor outside the call's tables";
            return err;
        }
        out.flops += row_flops(i);
        out.ins.push_back(i);
    }
    uint32_t s = 0;
    while (s < out.ins.size() && ins_kind(out.ins[s]) == K_SOURCE) s++;
    for (size_t n = s; n < out.ins.size(); n++)
        if (ins_kind(out.ins[n]) == K_SOURCE) {
            err.status = 3;
            err.message = "a source row follows other rows";
            return err;
        }
    out.sources = s;
    // dataflow over current planes: which are read before written (live-in), which written
    std::vector<uint8_t> state(P, 0);  // bit 0 written, bit 1 read-before-write
    auto read = [&](uint64_t p, uint64_t n) {
        for (uint64_t k = 0; k < n; k++)
            if (!(state[p + k] & 1)) state[p + k] |= 2;
    };
    auto write = [&](uint64_t p, uint64_t n) {
        for (uint64_t k = 0; k < n; k++) state[p + k] |= 1;
    };
    for (const Ins &i : out.ins) {
        switch (ins_kind(i)) {
        case K_CONTRIB: {
            int c0, c1, cd;
            contribution_shape(ins_op(i), &c0, &c1, &cd);
            read(i.a, c0);
            read(i.b, c1);
            if ((ins_flags(i) & F_FIRST) && !(ins_flags(i) & F_INIT)) read(i.c, cd);
            if (ins_flags(i) & F_LAST) write(i.c, cd);
            break;
        }
        case K_PROP: read(i.a, ins_op(i) == 9 ? 4 : 2); write(i.a, ins_op(i) == 9 ? 4 : 2); break;
        case K_IDENTITY: read(i.a, i.b); write(i.a, i.b); break;
        case K_CLEAR: write(i.a, i.b); break;
        case K_CLOSURE: read(i.a, i.s); read(i.b, i.s); break;
        case K_SOURCE: write(i.a, (i.y & 7) == 0 ? 1 : (i.y & 7) == 1 ? 2 : 4); break;
        }
    }
    // the program's needs: the largest reference of each kind
    Limits need{0, 0, 0, 0, 0};
    auto grow = [](uint64_t &n, uint64_t v) { n = std::max(n, v); };
    for (const Ins &i : out.ins) {
        int c0, c1, cd;
        switch (ins_kind(i)) {
        case K_CONTRIB:
            contribution_shape(ins_op(i), &c0, &c1, &cd);
            grow(need.current_planes, (uint64_t)i.a + c0);
            grow(need.current_planes, (uint64_t)i.b + c1);
            grow(need.current_planes, (uint64_t)i.c + cd);
            grow(need.scales, (uint64_t)i.s + 1);
            grow(need.factors, (uint64_t)i.x + 1);
            if (ins_op(i) == 6) grow(need.forms, (uint64_t)std::max(i.f & 0xffff, i.f >> 16) + 1);
            break;
        case K_PROP:
            grow(need.current_planes, (uint64_t)i.a + (ins_op(i) == 9 ? 4 : 2));
            grow(need.forms, (uint64_t)i.f + 1);
            grow(need.factors, (uint64_t)i.x + 1);
            break;
        case K_IDENTITY: grow(need.current_planes, (uint64_t)i.a + i.b); grow(need.factors, (uint64_t)i.x + 1); break;
        case K_CLEAR: grow(need.current_planes, (uint64_t)i.a + i.b); break;
        case K_CLOSURE:
            grow(need.current_planes, (uint64_t)std::max(i.a, i.b) + i.s);
            grow(need.amplitude_planes, (uint64_t)i.c + 1);
            grow(need.factors, std::max((uint64_t)i.x + 1, (uint64_t)i.y + i.s));
            break;
        case K_SOURCE:
            grow(need.current_planes, (uint64_t)i.a + ((i.y & 7) == 0 ? 1 : (i.y & 7) == 1 ? 2 : 4));
            grow(need.forms, (uint64_t)i.f + 1);
            grow(need.factors, (uint64_t)i.x + 1);
            grow(need.scales, (uint64_t)i.s + 1);
            break;
        }
    }
    out.need = need;
    out.reads_before_write.clear();
    out.writes.assign(P, 0);
    for (uint64_t p = 0; p < P; p++) {
        if (state[p] & 2) out.reads_before_write.push_back((uint32_t)p);
        out.writes[p] = state[p] & 1;
    }
    return err;
}

}  // namespace pacuda
