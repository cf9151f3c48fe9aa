// Test harness (CPU): the product's plan compiler and scheduler (pacuda_b200/csrc/program.cpp,
// schedule.cpp) driven from Python, for schedule statistics and for the CPU emulation of the
// on-chip executor's schedule in tests/test_schedule.py.
#include <stdint.h>
#include <string.h>

#include "../../pacuda_b200/csrc/program.h"
#include "../../pacuda_b200/csrc/schedule.h"

using namespace pacuda;

extern "C" {

// stats[0..8] = rows, tasks, levels, cur_slots, amp_slots, max_task_len, live-in groups, max tasks per
// level, peak live current slots
int schedule_stats(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                   uint32_t forms, uint32_t scales, uint32_t factors, uint32_t *stats) {
    Program p;
    Limits lim{planes, amps, forms, scales, factors};
    BuildError e = build_program(words, count, width, true, lim, p);
    if (e.status) return e.status;
    Schedule s;
    if (!build_schedule(p, planes, amps, s)) return -1;
    stats[0] = (uint32_t)p.ins.size();
    stats[1] = (uint32_t)s.task_first.size() - 1;
    stats[2] = (uint32_t)s.level_first.size() - 1;
    stats[3] = s.cur_slots;
    stats[4] = s.amp_slots;
    stats[5] = s.max_task_len;
    stats[6] = (uint32_t)s.loads.size() / 3;
    uint32_t mx = 0;
    for (size_t l = 0; l + 1 < s.level_first.size(); l++) mx = std::max(mx, s.level_first[l + 1] - s.level_first[l]);
    stats[7] = mx;
    stats[8] = s.peak_live;
    return 0;
}

// the program's instructions (the plan's row order, contribution runs grouped when `group`):
// count, then 8 u32 each
int program_export_order(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                         uint32_t forms, uint32_t scales, uint32_t factors, int group, uint32_t *n, uint32_t *ins) {
    Program p;
    Limits lim{planes, amps, forms, scales, factors};
    BuildError e = build_program(words, count, width, group != 0, lim, p);
    if (e.status) return e.status;
    *n = (uint32_t)p.ins.size();
    if (ins) memcpy(ins, p.ins.data(), p.ins.size() * sizeof(Ins));
    return 0;
}

// the program's instructions as the device runs them (contribution runs grouped)
int program_export(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                   uint32_t forms, uint32_t scales, uint32_t factors, uint32_t *n, uint32_t *ins) {
    return program_export_order(words, count, width, planes, amps, forms, scales, factors, 1, n, ins);
}

// build_program's status for a plan (0, or the runner's status code)
int program_status(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                   uint32_t forms, uint32_t scales, uint32_t factors) {
    Program p;
    Limits lim{planes, amps, forms, scales, factors};
    return build_program(words, count, width, true, lim, p).status;
}

// the schedule's arrays (for the emulator): sizes first (ins, tasks + 1, levels + 1, loads, amp planes)
int schedule_export(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                    uint32_t forms, uint32_t scales, uint32_t factors, uint32_t *sizes, uint32_t *ins,
                    uint32_t *task_first, uint32_t *level_first, uint32_t *loads, uint32_t *amp_planes,
                    uint32_t *slots) {
    Program p;
    Limits lim{planes, amps, forms, scales, factors};
    BuildError e = build_program(words, count, width, true, lim, p);
    if (e.status) return e.status;
    Schedule s;
    if (!build_schedule(p, planes, amps, s)) return -1;
    sizes[0] = (uint32_t)s.ins.size();
    sizes[1] = (uint32_t)s.task_first.size();
    sizes[2] = (uint32_t)s.level_first.size();
    sizes[3] = (uint32_t)s.loads.size();
    sizes[4] = (uint32_t)s.amp_planes.size();
    sizes[5] = s.cur_slots;
    sizes[6] = p.sources;
    if (ins) {
        memcpy(ins, s.ins.data(), s.ins.size() * sizeof(Ins));
        memcpy(task_first, s.task_first.data(), s.task_first.size() * 4);
        memcpy(level_first, s.level_first.data(), s.level_first.size() * 4);
        memcpy(loads, s.loads.data(), s.loads.size() * 4);
        memcpy(amp_planes, s.amp_planes.data(), s.amp_planes.size() * 4);
        (void)slots;
    }
    return 0;
}
}

extern "C" {
// the schedule in reduction-term mode (use_terms with the reduction offsets[outputs + 1], planes):
// sizes = ins, tasks + 1, levels + 1, applied (0/1), terms, cur_slots; arrays as schedule_export
int schedule_export_terms(const uint64_t *words, uint32_t count, const uint8_t *width, uint32_t planes, uint32_t amps,
                          uint32_t forms, uint32_t scales, uint32_t factors, const uint32_t *offsets,
                          const uint32_t *red_planes, uint32_t outputs, uint32_t *sizes, uint32_t *ins,
                          uint32_t *task_first, uint32_t *level_first) {
    Program p;
    Limits lim{planes, amps, forms, scales, factors};
    BuildError e = build_program(words, count, width, true, lim, p);
    if (e.status) return e.status;
    Schedule s;
    if (!build_schedule(p, planes, amps, s)) return -1;
    bool applied = use_terms(s, offsets, red_planes, outputs, amps);
    sizes[0] = (uint32_t)s.ins.size();
    sizes[1] = (uint32_t)s.task_first.size();
    sizes[2] = (uint32_t)s.level_first.size();
    sizes[3] = applied;
    sizes[4] = s.terms;
    sizes[5] = s.cur_slots;
    if (ins) {
        memcpy(ins, s.ins.data(), s.ins.size() * sizeof(Ins));
        memcpy(task_first, s.task_first.data(), s.task_first.size() * 4);
        memcpy(level_first, s.level_first.data(), s.level_first.size() * 4);
    }
    return 0;
}
}
