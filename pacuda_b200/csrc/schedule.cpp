// Host scheduling of a plan for the on-chip executor (see schedule.h).
#include "schedule.h"

#include <algorithm>
#include <map>
#include <numeric>
#include <queue>

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
    uint32_t amplitude = ~0u;           // closures: their amplitude plane
    std::vector<uint32_t> amplitudes;   // closures fused into a current's task: their amplitudes
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

    // ---- propagators fused into the run of their current ----
    // A propagator acts in place on the current a destination run wrote. When no task between
    // the run and the propagator (in program order) reads or writes that current, the propagator
    // can follow the run at once: the run's task applies it, and it needs no level of its own.
    {
        std::vector<std::vector<Range>> touched(tasks.size());
        for (size_t ti = 0; ti < tasks.size(); ti++) {
            std::vector<Range> r, w;
            for (const Ins &i : tasks[ti].ins) access(i, r, w);
            touched[ti] = r;
            touched[ti].insert(touched[ti].end(), w.begin(), w.end());
        }
        auto overlaps = [](const std::vector<Range> &v, uint32_t first, uint32_t count) {
            for (const Range &x : v)
                if (x.first < first + count && first < x.first + x.count) return true;
            return false;
        };
        std::vector<uint8_t> gone(tasks.size(), 0);
        for (size_t ti = 0; ti < tasks.size(); ti++) {
            if (tasks[ti].ins.size() != 1 || ins_kind(tasks[ti].ins[0]) != K_PROP) continue;
            const Ins &prop = tasks[ti].ins[0];
            const uint32_t m = ins_op(prop) == 9 ? 4 : 2;
            for (size_t tj = ti; tj-- > 0;) {
                if (gone[tj] || !overlaps(touched[tj], prop.a, m)) continue;
                Task &run = tasks[tj];
                const Ins &last = run.ins.back();
                int c0, c1, cd;
                contribution_shape(ins_op(last), &c0, &c1, &cd);
                if (ins_kind(last) == K_CONTRIB && (ins_flags(last) & F_LAST) && last.c == prop.a && (uint32_t)cd == m) {
                    run.ins.push_back(prop);
                    gone[ti] = 1;
                }
                break;  // the nearest task that touches the current decides
            }
        }
        std::vector<Task> kept;
        for (size_t ti = 0; ti < tasks.size(); ti++)
            if (!gone[ti]) kept.push_back(std::move(tasks[ti]));
        tasks.swap(kept);
    }

    // ---- closures fused into the task of their closing current ----
    // A closing current read by nothing but closures, whose amplitudes receive no other closure,
    // is computed, closed and forgotten by one task: the closures read its sums in registers and
    // it needs no slot. (Its values still go to the global arena in the C ABI's mode.)
    std::vector<uint8_t> in_register(G, 0);
    {
        std::vector<int> closure_tasks_of(A, 0);
        for (const Task &t : tasks)
            if (t.amplitude != ~0u) closure_tasks_of[t.amplitude]++;
        // per group: its tasks that read or write it
        std::vector<std::vector<uint32_t>> readers(G), writers(G);
        for (uint32_t ti = 0; ti < tasks.size(); ti++) {
            std::vector<Range> r, w;
            for (const Ins &i : tasks[ti].ins) access(i, r, w);
            for (const Range &x : r)
                for (uint32_t k = 0; k < x.count; k++) {
                    auto &v = readers[group_of[x.first + k]];
                    if (v.empty() || v.back() != ti) v.push_back(ti);
                }
            for (const Range &x : w)
                for (uint32_t k = 0; k < x.count; k++) {
                    auto &v = writers[group_of[x.first + k]];
                    if (v.empty() || v.back() != ti) v.push_back(ti);
                }
        }
        std::vector<uint8_t> merged(tasks.size(), 0);
        for (uint32_t g = 0; g < G; g++) {
            if (writers[g].size() != 1 || readers[g].empty()) continue;
            uint32_t pt = writers[g][0];
            Task &prod = tasks[pt];
            const Ins &last = prod.ins.back();
            int c0, c1, cd;
            if (ins_kind(last) != K_CONTRIB || !(ins_flags(last) & F_LAST)) continue;
            contribution_shape(ins_op(last), &c0, &c1, &cd);
            if (last.c != gbase[g] || (uint32_t)cd != gsize[g] || !(ins_flags(prod.ins.front()) & F_INIT)) continue;
            bool ok = true;
            for (const Ins &i : prod.ins) {  // every row of the run writes the same components
                int a0, a1, ad;
                contribution_shape(ins_op(i), &a0, &a1, &ad);
                if (ins_kind(i) != K_CONTRIB || ad != cd) ok = false;
            }
            for (uint32_t rt : readers[g]) {
                const Task &t = tasks[rt];
                if (rt == pt || t.amplitude == ~0u || closure_tasks_of[t.amplitude] != 1 || rt < pt) ok = false;
                for (const Ins &i : t.ins)
                    if (ins_kind(i) != K_CLOSURE || i.a != gbase[g] || i.s > gsize[g] ||
                        (i.b < gbase[g] + gsize[g] && i.b + i.s > gbase[g]))
                        ok = false;
            }
            if (!ok) continue;
            for (uint32_t rt : readers[g]) {
                for (Ins i : tasks[rt].ins) {
                    i.head |= F_ACC0 << 8;
                    prod.ins.push_back(i);
                }
                prod.amplitudes.push_back(tasks[rt].amplitude);
                merged[rt] = 1;
            }
            for (Ins &i : prod.ins)
                if (ins_kind(i) == K_CONTRIB && (ins_flags(i) & F_LAST)) i.head |= F_NOSTORE << 8;
            in_register[g] = 1;
        }
        std::vector<Task> kept;
        for (uint32_t ti = 0; ti < tasks.size(); ti++)
            if (!merged[ti]) kept.push_back(std::move(tasks[ti]));
        tasks.swap(kept);
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
        for (uint32_t a : t.amplitudes) lvl = std::max(lvl, std::max(alw[a], alr[a]) + 1);
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
        for (uint32_t a : t.amplitudes) alw[a] = lvl;
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
    // Spread placement. A block of one point reads one slot per lane, 16 bytes at a time; eight
    // lanes share a shared-memory wavefront over eight 16-byte bank groups, and values packed at
    // slots 4m (the 4-component currents) fall into two of them. So, when no group is wider than
    // kWindow slots, no group crosses a multiple of kWindow (a group that would starts at the next
    // one), and each window of kWindow slots is followed by one unused slot: window w starts at
    // 13w, so the windows' values start in all eight bank groups. (12 = 4 x 3 = 6 x 2 packs the
    // 4- and 6-slot values of the gluon plans without loss; 8 % more slots.)
    constexpr uint32_t kWindow = 12;
    uint32_t widest = 0;
    for (uint32_t g = 0; g < G; g++)
        if (!in_register[g]) widest = std::max(widest, gsize[g]);
    const bool spread = widest <= kWindow;
    // the first start at or after s where z slots cross no multiple of kWindow
    auto start_at = [&](uint32_t s, uint32_t z) -> uint32_t {
        return !spread || z == 0 || s / kWindow == (s + z - 1) / kWindow ? s : (s + kWindow - 1) / kWindow * kWindow;
    };
    for (uint32_t g : order) {
        if (in_register[g]) continue;  // kept in a task's registers
        // a slot is reused only after the last level that touches its previous occupant
        while (!active.empty() && active.begin()->first < gfirst[g]) {
            release(active.begin()->second.first, active.begin()->second.second);
            active.erase(active.begin());
        }
        const uint32_t z = gsize[g];
        uint32_t slot = ~0u;
        for (auto it = free.begin(); it != free.end(); ++it) {
            const uint32_t s = it->first, size = it->second, a = start_at(s, z);
            if (a + z <= s + size) {
                free.erase(it);
                if (a > s) free.emplace(s, a - s);
                if (a + z < s + size) free.emplace(a + z, s + size - a - z);
                slot = a;
                break;
            }
        }
        if (slot == ~0u) {
            const uint32_t a = start_at(top, z);
            if (a > top) release(top, a - top);
            slot = a;
            top = a + z;
        }
        gslot[g] = slot;
        active.emplace(glast[g], std::make_pair(slot, z));
    }
    if (spread) {
        auto place = [](uint32_t s) { return (kWindow + 1) * (s / kWindow) + s % kWindow; };
        for (uint32_t g = 0; g < G; g++)
            if (!in_register[g]) gslot[g] = place(gslot[g]);
        top = top ? place(top - 1) + 1 : 0;
    }
    out.cur_slots = top;
    {
        int levels_n = 0;
        for (uint32_t g = 0; g < G; g++) levels_n = std::max(levels_n, glast[g] + 1);
        std::vector<uint32_t> live((size_t)std::max(levels_n, 1), 0);
        for (uint32_t g = 0; g < G; g++)
            if (!in_register[g] && glast[g] >= 0)
                for (int l = gfirst[g]; l <= glast[g]; l++) live[l] += gsize[g];
        out.peak_live = *std::max_element(live.begin(), live.end());
    }
    auto slot_of = [&](uint32_t plane) {
        uint32_t g = group_of[plane];
        return in_register[g] ? 0u : gslot[g] + (plane - gbase[g]);
    };
    for (uint32_t g = 0; g < G; g++)
        if (live_in[g]) {
            out.loads.push_back(gbase[g]);
            out.loads.push_back(gslot[g]);
            out.loads.push_back(gsize[g]);
        }
    // amplitude slots: one per amplitude a closure accumulates into, for the whole run
    out.amp_slot_of.assign(A, ~0u);
    for (const Task &t : tasks)
        for (const Ins &i : t.ins)
            if (ins_kind(i) == K_CLOSURE && out.amp_slot_of[i.c] == ~0u) {
                out.amp_slot_of[i.c] = (uint32_t)out.amp_planes.size();
                out.amp_planes.push_back(i.c);
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
        uint32_t cost = 0;
        for (const Ins &i : tasks[t].ins) cost += ins_flops(i) + 8;  // + its fetch and decode
        out.task_cost.push_back(cost);
    }
    return true;
}

void lane_order(const Schedule &s, uint32_t lanes, std::vector<uint32_t> &order, std::vector<uint32_t> &level_first) {
    const uint32_t L = lanes;
    order.clear();
    level_first.assign(1, 0);
    for (size_t lv = 0; lv + 1 < s.level_first.size(); lv++) {
        std::vector<uint32_t> ts;
        for (uint32_t t = s.level_first[lv]; t < s.level_first[lv + 1]; t++) ts.push_back(t);
        std::stable_sort(ts.begin(), ts.end(), [&](uint32_t x, uint32_t y) { return s.task_cost[x] > s.task_cost[y]; });
        // longest first onto the least loaded lane (ties: the lowest lane)
        std::vector<std::vector<uint32_t>> lane(L);
        typedef std::pair<uint64_t, uint32_t> Load;
        std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
        for (uint32_t l = 0; l < L; l++) heap.push({0, l});
        for (uint32_t t : ts) {
            Load top = heap.top();
            heap.pop();
            lane[top.second].push_back(t);
            heap.push({top.first + s.task_cost[t], top.second});
        }
        size_t rounds = 0;
        for (auto &v : lane) rounds = std::max(rounds, v.size());
        for (size_t r = 0; r < rounds; r++)
            for (uint32_t l = 0; l < L; l++) order.push_back(r < lane[l].size() ? lane[l][r] : ~0u);
        level_first.push_back((uint32_t)order.size());
    }
}

bool use_terms(Schedule &s, const uint32_t *offsets, const uint32_t *planes, uint32_t outputs, uint32_t amplitude_planes) {
    const uint32_t T = offsets[outputs];
    if (T >= 0xffff) return false;
    std::vector<uint32_t> term_of(amplitude_planes, 0xffff), rows(amplitude_planes, 0);
    for (uint32_t k = 0; k < T; k++) {
        if (planes[k] >= amplitude_planes || term_of[planes[k]] != 0xffff) return false;  // one term per amplitude
        term_of[planes[k]] = k;
    }
    for (const Ins &i : s.ins)
        if (ins_kind(i) == K_CLOSURE && ++rows[i.f] > 1) return false;  // (a closure's f is its amplitude plane)
    for (Ins &i : s.ins)
        if (ins_kind(i) == K_CLOSURE) {
            i.head |= F_TERM << 8;
            i.c = term_of[i.f];
        }
    s.terms = T;
    s.amp_slots = 0;
    s.amp_planes.clear();
    return true;
}

}  // namespace pacuda
