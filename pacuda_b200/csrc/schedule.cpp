// Host scheduling of a plan for the on-chip executor (see schedule.h).
#include "schedule.h"

#include <algorithm>
#include <map>
#include <numeric>

namespace pacuda {
namespace {

struct Range {
    uint32_t first, count;
};

int source_components(uint32_t code) {
    uint32_t family = code & 7;
    return family == 0 ? 1 : family == 1 ? 2 : 4;
}

// the current-plane ranges an instruction reads and writes (the reference's semantics)
void access(const Ins &i, std::vector<Range> &reads, std::vector<Range> &writes) {
    int c0, c1, cd;
    switch (ins_kind(i)) {
    case K_CONTRIB:
        contribution_shape(ins_op(i), &c0, &c1, &cd);
        reads.push_back({i.a, (uint32_t)c0});
        reads.push_back({i.b, (uint32_t)c1});
        if ((ins_flags(i) & F_FIRST) && !(ins_flags(i) & F_INIT)) reads.push_back({i.c, (uint32_t)cd});
        if (ins_flags(i) & F_LAST) writes.push_back({i.c, (uint32_t)cd});
        break;
    case K_PROP: {
        uint32_t m = ins_op(i) == 9 ? 4 : 2;
        reads.push_back({i.a, m});
        writes.push_back({i.a, m});
        break;
    }
    case K_IDENTITY: reads.push_back({i.a, i.b}); writes.push_back({i.a, i.b}); break;
    case K_CLEAR: writes.push_back({i.a, i.b}); break;
    case K_CLOSURE: reads.push_back({i.a, i.s}); reads.push_back({i.b, i.s}); break;
    case K_SOURCE: writes.push_back({i.a, (uint32_t)source_components(i.y)}); break;
    }
}

struct Uf {
    std::vector<uint32_t> parent;
    explicit Uf(size_t n) : parent(n) { std::iota(parent.begin(), parent.end(), 0u); }
    uint32_t find(uint32_t x) {
        while (parent[x] != x) x = parent[x] = parent[parent[x]];
        return x;
    }
    void join(uint32_t a, uint32_t b) {
        a = find(a);
        b = find(b);
        if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
};

struct Task {
    std::vector<Ins> ins;
    int level = 0;
    bool source = false;
    uint32_t amplitude = ~0u;  // closures: their amplitude plane
};

}  // namespace

bool build_schedule(const Program &p, uint32_t P, uint32_t A, Schedule &out) {
    out = Schedule();
    const std::vector<Ins> &in = p.ins;
    // ---- plane groups: operands read or written as a whole share a group ----
    Uf uf(P + 1);
    std::vector<uint8_t> touched(P, 0), structural(P, 0);
    for (const Ins &i : in) {
        std::vector<Range> r, w;
        access(i, r, w);
        bool piecewise = ins_kind(i) == K_IDENTITY || ins_kind(i) == K_CLEAR;
        for (auto *v : {&r, &w})
            for (const Range &x : *v) {
                for (uint32_t k = 0; k < x.count; k++) {
                    touched[x.first + k] = 1;
                    if (!piecewise) structural[x.first + k] = 1;
                }
                if (!piecewise)
                    for (uint32_t k = 1; k < x.count; k++) uf.join(x.first, x.first + k);
            }
    }
    // planes only cleared or scaled: consecutive ones of one range form a group
    for (const Ins &i : in)
        if (ins_kind(i) == K_IDENTITY || ins_kind(i) == K_CLEAR)
            for (uint32_t k = 1; k < i.b; k++)
                if (!structural[i.a + k] && !structural[i.a + k - 1]) uf.join(i.a + k - 1, i.a + k);
    std::vector<uint32_t> group_of(P, ~0u), gbase, gsize;
    for (uint32_t q = 0; q < P; q++) {
        if (!touched[q]) continue;
        uint32_t root = uf.find(q);
        if (group_of[root] == ~0u) {
            group_of[root] = (uint32_t)gbase.size();
            gbase.push_back(q);
            gsize.push_back(0);
        }
        group_of[q] = group_of[root];
        gsize[group_of[q]] = q - gbase[group_of[q]] + 1;
    }
    const uint32_t G = (uint32_t)gbase.size();

    // ---- tasks ----
    // The sources run first, from the f64 forms, at level 0 (the kernel turns the forms into the
    // kind's layout after them). Sources that write overlapping planes form one task, so that
    // they keep their order; others are one task each.
    std::vector<Task> tasks;
    bool sources_overlap = false;
    {
        std::vector<uint8_t> hit(P, 0);
        for (uint32_t s = 0; s < p.sources && !sources_overlap; s++)
            for (int k = 0; k < source_components(in[s].y); k++) {
                if (hit[in[s].a + k]) sources_overlap = true;
                hit[in[s].a + k] = 1;
            }
    }
    size_t n = 0;
    if (sources_overlap && p.sources) {
        Task t;
        t.source = true;
        for (; n < p.sources; n++) t.ins.push_back(in[n]);
        tasks.push_back(t);
    }
    while (n < in.size()) {
        const Ins &i = in[n];
        Task t;
        uint32_t kind = ins_kind(i);
        if (kind == K_SOURCE) {
            t.ins.push_back(i);
            t.source = true;
            n++;
        } else if (kind == K_CONTRIB) {
            // a destination's run: F_FIRST .. F_LAST (the program marks consecutive rows of one
            // destination)
            t.ins.push_back(in[n++]);
            while (!(ins_flags(t.ins.back()) & F_LAST) && n < in.size() && ins_kind(in[n]) == K_CONTRIB &&
                   !(ins_flags(in[n]) & F_FIRST))
                t.ins.push_back(in[n++]);
            int c0, c1, cd;
            contribution_shape(ins_op(t.ins.back()), &c0, &c1, &cd);
            if (n < in.size() && ins_kind(in[n]) == K_PROP && in[n].a == i.c &&
                (uint32_t)cd == (ins_op(in[n]) == 9 ? 4u : 2u))
                t.ins.push_back(in[n++]);
        } else if (kind == K_IDENTITY || kind == K_CLEAR) {
            // one task per group the range covers
            uint32_t q = i.a, end = i.a + i.b;
            while (q < end) {
                uint32_t g = group_of[q];
                uint32_t stop = std::min(end, gbase[g] + gsize[g]);
                Task piece;
                Ins c = i;
                c.a = q;
                c.b = stop - q;
                piece.ins.push_back(c);
                tasks.push_back(piece);
                q = stop;
            }
            n++;
            continue;
        } else if (kind == K_CLOSURE) {
            t.amplitude = i.c;
            t.ins.push_back(in[n++]);
            while (n < in.size() && ins_kind(in[n]) == K_CLOSURE && in[n].c == i.c) t.ins.push_back(in[n++]);
        } else {
            t.ins.push_back(in[n++]);
        }
        tasks.push_back(t);
    }

    // ---- levels ----
    std::vector<int> lw(P, -1), lr(P, -1), alw(A, -1), alr(A, -1);
    int levels = 1;
    for (Task &t : tasks) {
        std::vector<Range> r, w;
        for (const Ins &i : t.ins) access(i, r, w);
        int lvl = t.source ? 0 : 1;  // sources: 0 (their overlaps are inside one task)
        for (const Range &x : r)
            for (uint32_t k = 0; k < x.count; k++) lvl = std::max(lvl, lw[x.first + k] + 1);
        for (const Range &x : w)
            for (uint32_t k = 0; k < x.count; k++)
                lvl = std::max(lvl, std::max(lw[x.first + k], lr[x.first + k]) + 1);
        if (t.amplitude != ~0u) lvl = std::max(lvl, std::max(alw[t.amplitude], alr[t.amplitude]) + 1);
        if (t.source) lvl = 0;
        t.level = lvl;
        for (const Range &x : r)
            for (uint32_t k = 0; k < x.count; k++) lr[x.first + k] = std::max(lr[x.first + k], lvl);
        for (const Range &x : w)
            for (uint32_t k = 0; k < x.count; k++) {
                lw[x.first + k] = lvl;
                lr[x.first + k] = -1;
            }
        if (t.amplitude != ~0u) alw[t.amplitude] = lvl;
        levels = std::max(levels, lvl + 1);
    }

    // ---- the last writer of each plane (its values go to the global arena in the ABI's mode) ----
    std::vector<std::pair<uint32_t, uint32_t>> last(P, {~0u, ~0u});  // plane -> (task, instruction)
    for (uint32_t t = 0; t < tasks.size(); t++)
        for (uint32_t k = 0; k < tasks[t].ins.size(); k++) {
            std::vector<Range> r, w;
            access(tasks[t].ins[k], r, w);
            for (const Range &x : w)
                for (uint32_t q = 0; q < x.count; q++) last[x.first + q] = {t, k};
        }
    for (uint32_t q = 0; q < P; q++)
        if (last[q].first != ~0u) tasks[last[q].first].ins[last[q].second].head |= F_WB << 8;

    // ---- liveness and slots ----
    std::vector<int> gfirst(G, 1 << 30), glast(G, -1);
    for (const Task &t : tasks) {
        std::vector<Range> r, w;
        for (const Ins &i : t.ins) access(i, r, w);
        for (auto *v : {&r, &w})
            for (const Range &x : *v)
                for (uint32_t k = 0; k < x.count; k++) {
                    uint32_t g = group_of[x.first + k];
                    gfirst[g] = std::min(gfirst[g], t.level);
                    glast[g] = std::max(glast[g], t.level);
                }
    }
    std::vector<uint8_t> live_in(G, 0);
    for (uint32_t q : p.reads_before_write) {
        uint32_t g = group_of[q];
        live_in[g] = 1;
        gfirst[g] = 0;
    }
    std::vector<uint32_t> order(G);
    std::iota(order.begin(), order.end(), 0u);
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return gfirst[x] != gfirst[y] ? gfirst[x] < gfirst[y] : gsize[x] > gsize[y];
    });
    std::vector<uint32_t> gslot(G, 0);
    std::multimap<int, std::pair<uint32_t, uint32_t>> active;  // end level -> (slot, size)
    std::map<uint32_t, uint32_t> free;                          // slot -> size
    uint32_t top = 0;
    auto release = [&](uint32_t s, uint32_t z) {
        auto it = free.emplace(s, z).first;
        auto next = std::next(it);
        if (next != free.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free.erase(next);
        }
        if (it != free.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free.erase(it);
            }
        }
    };
    for (uint32_t g : order) {
        // a slot is reused only after the last level that touches its previous occupant
        while (!active.empty() && active.begin()->first < gfirst[g]) {
            release(active.begin()->second.first, active.begin()->second.second);
            active.erase(active.begin());
        }
        uint32_t slot = ~0u;
        for (auto it = free.begin(); it != free.end(); ++it)
            if (it->second >= gsize[g]) {
                slot = it->first;
                uint32_t rest = it->second - gsize[g];
                free.erase(it);
                if (rest) free.emplace(slot + gsize[g], rest);
                break;
            }
        if (slot == ~0u) {
            slot = top;
            top += gsize[g];
        }
        gslot[g] = slot;
        active.emplace(glast[g], std::make_pair(slot, gsize[g]));
    }
    out.cur_slots = top;
    auto slot_of = [&](uint32_t plane) { return gslot[group_of[plane]] + (plane - gbase[group_of[plane]]); };
    for (uint32_t g = 0; g < G; g++)
        if (live_in[g]) {
            out.loads.push_back(gbase[g]);
            out.loads.push_back(gslot[g]);
            out.loads.push_back(gsize[g]);
        }
    // amplitude slots: one per amplitude a closure accumulates into, for the whole run
    out.amp_slot_of.assign(A, ~0u);
    for (const Task &t : tasks)
        if (t.amplitude != ~0u && out.amp_slot_of[t.amplitude] == ~0u) {
            out.amp_slot_of[t.amplitude] = (uint32_t)out.amp_planes.size();
            out.amp_planes.push_back(t.amplitude);
        }
    out.amp_slots = (uint32_t)out.amp_planes.size();

    // ---- emit: levels in order; within a level the tasks sorted by their ops ----
    std::vector<uint32_t> idx(tasks.size());
    std::iota(idx.begin(), idx.end(), 0u);
    auto signature = [&](const Task &t) {
        uint64_t h = 1469598103934665603ull;
        for (const Ins &i : t.ins) h = (h ^ (i.head & 0x7ff)) * 1099511628211ull;
        return h;
    };
    std::vector<uint64_t> sig(tasks.size());
    for (size_t t = 0; t < tasks.size(); t++) sig[t] = signature(tasks[t]);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
        if (tasks[x].level != tasks[y].level) return tasks[x].level < tasks[y].level;
        if (tasks[x].ins.size() != tasks[y].ins.size()) return tasks[x].ins.size() > tasks[y].ins.size();
        return sig[x] < sig[y];
    });
    out.level_first.assign(levels + 1, 0);
    for (uint32_t t : idx) out.level_first[tasks[t].level + 1]++;
    for (int l = 0; l < levels; l++) out.level_first[l + 1] += out.level_first[l];
    out.task_first.push_back(0);
    for (uint32_t t : idx) {
        for (Ins i : tasks[t].ins) {
            uint32_t kind = ins_kind(i);
            switch (kind) {
            case K_CONTRIB: i.y = i.c; i.a = slot_of(i.a); i.b = slot_of(i.b); i.c = slot_of(i.c); break;
            case K_PROP: i.y = i.a; i.a = slot_of(i.a); break;
            case K_IDENTITY:
            case K_CLEAR: i.y = i.a; i.a = slot_of(i.a); break;
            case K_CLOSURE: i.f = i.c; i.a = slot_of(i.a); i.b = slot_of(i.b); i.c = out.amp_slot_of[i.c]; break;
            case K_SOURCE: i.c = i.a; i.a = slot_of(i.a); break;
            }
            out.ins.push_back(i);
        }
        out.task_first.push_back((uint32_t)out.ins.size());
        out.max_task_len = std::max<uint32_t>(out.max_task_len, (uint32_t)tasks[t].ins.size());
    }
    return true;
}

}  // namespace pacuda
