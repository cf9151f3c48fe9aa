// Host compilation of a plan's words into the device instruction stream.
//
// decode: the row layout of runner/recurrence_runner.cu:10-36 (fields of variable width after
// a 4-bit op; op 14 followed by its data words), as that file's `decode` (:920-975) and
// convert/src/program.rs (:60-114) read it. The sort: a run of contribution rows whose
// destinations do not overlap and that reads none of them is stably sorted by destination
// (:980-1007), which keeps every destination's own order of rows and so its value bit for bit.
// The F_FIRST / F_LAST flags mark a destination's run of rows so that its sum stays in
// registers (:1017-1054).
#include "program.h"

#include <algorithm>
#include <unordered_map>

namespace pacuda {

void contribution_shape(int op, int *c0, int *c1, int *cd) {
    *c0 = op == 4 ? 6 : (op == 5 || op == 6) ? 4 : 2;
    *c1 = 4;
    *cd = (op == 4 || op == 6) ? 4 : op == 5 ? 6 : 2;
}

bool decode_rows(const uint64_t *words, uint32_t count, const uint8_t *width, std::vector<Row> &rows,
                 std::vector<uint32_t> &binding_data) {
    rows.clear();
    binding_data.clear();
    for (uint32_t n = 0; n < count; n++) {
        uint64_t w = words[n];
        if ((w & 15) == 14) {
            Row r{};
            r.op = 14;
            r.f[0] = (uint32_t)(w >> 4) & 0xffff;
            r.f[1] = (uint32_t)(w >> 20) & 0xff;
            r.f[2] = (uint32_t)(w >> 28) & 0xff;
            r.f[3] = (uint32_t)(w >> 36) & 1;
            uint32_t codes = r.f[1] + r.f[2];
            r.data_first = (uint32_t)binding_data.size();
            r.data_count = codes;
            for (uint32_t k = 0; k < codes; k++) {
                uint64_t d = n + 1 + k / 2 < count ? words[n + 1 + k / 2] : 0;
                binding_data.push_back((uint32_t)(k % 2 ? d >> 32 : d));
            }
            n += (codes + 1) / 2;
            rows.push_back(r);
            continue;
        }
        bool wide = false;
        auto take = [&](int bits) -> uint32_t {
            if (bits > 32) { wide = true; return 0; }
            uint32_t v = (uint32_t)(w & ((1ull << bits) - 1));
            w >>= bits;
            return v;
        };
        Row r{};
        r.op = (int)take(4);
        const int P = width[WP], A = width[WA], F = width[WF], X = width[WX], S = width[WS], K = width[WK];
        int fields[8] = {0}, nf = 0;
        switch (r.op) {
        case 1: fields[0] = P; fields[1] = P; nf = 2; break;
        case 2: case 3: case 4: case 5: case 6: {
            int f[8] = {1, S, P, P, P, F, F, X};
            std::copy(f, f + 8, fields);
            nf = 8;
            break;
        }
        case 7: case 8: case 9: fields[0] = P; fields[1] = F; fields[2] = X; nf = 3; break;
        case 10: fields[0] = P; fields[1] = K; fields[2] = X; nf = 3; break;
        case 11: {
            int f[6] = {P, P, A, X, X, K};
            std::copy(f, f + 6, fields);
            nf = 6;
            break;
        }
        case 12: {
            int f[5] = {P, F, X, S, 10};
            std::copy(f, f + 5, fields);
            nf = 5;
            break;
        }
        case 13: {
            int f[7] = {1, P, P, P, F, F, X};
            std::copy(f, f + 7, fields);
            nf = 7;
            break;
        }
        default: return false;  // ops 0 and 15 do not exist
        }
        for (int k = 0; k < nf; k++) r.f[k] = take(fields[k]);
        if (wide) return false;
        rows.push_back(r);
    }
    return true;
}

void sort_contribution_runs(std::vector<Row> &rows) {
    size_t n = 0;
    while (n < rows.size()) {
        if (rows[n].op < 2 || rows[n].op > 6) { n++; continue; }
        size_t end = n;
        while (end < rows.size() && rows[end].op >= 2 && rows[end].op <= 6) end++;
        std::unordered_map<uint32_t, uint32_t> owner;  // component -> its destination's base
        bool safe = true;
        for (size_t k = n; k < end && safe; k++) {
            int c0, c1, cd;
            contribution_shape(rows[k].op, &c0, &c1, &cd);
            for (int q = 0; q < cd; q++) {
                auto it = owner.emplace(rows[k].f[4] + q, rows[k].f[4]);
                if (it.first->second != rows[k].f[4]) safe = false;
            }
        }
        for (size_t k = n; k < end && safe; k++) {
            int c0, c1, cd;
            contribution_shape(rows[k].op, &c0, &c1, &cd);
            for (int q = 0; q < c0 && safe; q++) safe = !owner.count(rows[k].f[2] + q);
            for (int q = 0; q < c1 && safe; q++) safe = !owner.count(rows[k].f[3] + q);
        }
        if (safe)
            std::stable_sort(rows.begin() + n, rows.begin() + end,
                             [](const Row &x, const Row &y) { return x.f[4] < y.f[4]; });
        n = end;
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
    for (int k = 0; k < 6; k++)
        if (width[k] > 32) {
            err.status = 2;
            err.message = "a field width above 32 bits";
            return err;
        }
    if (!decode_rows(words, count, width, rows, binding_data)) {
        err.status = 2;
        err.message = "a word with an op outside 1..14";
        return err;
    }
    for (const Row &r : rows)
        if (r.op == 13 || r.op == 14) {
            // as a runner built without generated symjit kernels (recurrence_runner.cu:1141-1145)
            err.status = 3;
            err.message = "a symjit row, but this runner has no symjit kernels";
            return err;
        }
    if (sort) sort_contribution_runs(rows);
    out.ins.clear();
    out.ins.reserve(rows.size());
    out.flops = 0;
    uint64_t P = lim.current_planes;
    for (size_t n = 0; n < rows.size(); n++) {
        const Row &r = rows[n];
        const uint32_t *f = r.f;
        Ins i{};
        bool ok = true;
        if (r.op >= 2 && r.op <= 6) {
            bool first = n == 0 || rows[n - 1].op < 2 || rows[n - 1].op > 6 || rows[n - 1].f[4] != f[4];
            bool last = n + 1 == rows.size() || rows[n + 1].op < 2 || rows[n + 1].op > 6 || rows[n + 1].f[4] != f[4];
            i = make(K_CONTRIB, r.op, (f[0] ? F_INIT : 0) | (first ? F_FIRST : 0) | (last ? F_LAST : 0), 0);
            i.s = f[1]; i.a = f[2]; i.b = f[3]; i.c = f[4]; i.x = f[7];
            // the forms are read by op 6 only (a form index must fit 16 bits here)
            i.f = r.op == 6 ? ((f[5] & 0xffff) | (f[6] << 16)) : 0;
            int c0, c1, cd;
            contribution_shape(r.op, &c0, &c1, &cd);
            ok = within(f[2], c0, P) && within(f[3], c1, P) && within(f[4], cd, P) && f[1] < lim.scales &&
                 f[7] < lim.factors &&
                 (r.op != 6 || (f[5] < lim.forms && f[6] < lim.forms && f[5] < 65536 && f[6] < 65536));
        } else if (r.op == 1) {
            i = make(K_CLEAR, 1, 0, 0);
            i.a = f[0]; i.b = f[1];
            ok = within(f[0], f[1], P);
        } else if (r.op >= 7 && r.op <= 9) {
            i = make(K_PROP, r.op, 0, 0);
            i.a = f[0]; i.f = f[1]; i.x = f[2];
            ok = within(f[0], r.op == 9 ? 4 : 2, P) && f[1] < lim.forms && f[2] < lim.factors;
        } else if (r.op == 10) {
            i = make(K_IDENTITY, 10, 0, 0);
            i.a = f[0]; i.b = f[1]; i.x = f[2];
            ok = within(f[0], f[1], P) && f[2] < lim.factors;
        } else if (r.op == 11) {
            i = make(K_CLOSURE, 11, 0, 0);
            i.a = f[0]; i.b = f[1]; i.c = f[2]; i.x = f[3]; i.y = f[4];
            i.s = f[5];  // the component count
            ok = within(f[0], f[5], P) && within(f[1], f[5], P) && f[2] < lim.amplitude_planes && f[3] < lim.factors &&
                 within(f[4], f[5], lim.factors);
        } else {  // 12
            i = make(K_SOURCE, 12, 0, 0);
            i.a = f[0]; i.f = f[1]; i.x = f[2]; i.s = f[3]; i.y = f[4];
            int comps = (f[4] & 7) == 0 ? 1 : (f[4] & 7) == 1 ? 2 : 4;
            ok = within(f[0], comps, P) && f[1] < lim.forms && f[2] < lim.factors && f[3] < lim.scales;
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
