// The on-chip schedule of a plan: its rows grouped into tasks, the tasks into dataflow levels,
// and its current planes packed into shared-memory slots by liveness.
//
// A task is what one lane runs for one point with its sums in registers: a source row, a
// destination's run of contribution rows (F_FIRST .. F_LAST) with the propagator that
// follows it on the same current, a propagator, an identity or clear over one current, or a
// destination amplitude's consecutive closures. Tasks of one level read nothing another task of
// that level writes, so the lanes of a point run them in any order; each current's and each
// amplitude's rows keep their order, so every value is the one the row order gives, bit for bit.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "program.h"

namespace pacuda {

enum : uint32_t {
    F_WB = 8,        // the instruction's written values also go to the global arena
    F_ACC0 = 16,     // a closure whose parent 0 is the task's sums (its closing current, in registers)
    F_NOSTORE = 32,  // a destination run's last row keeps its sums in registers (no slot)
    F_TERM = 64,     // a closure that makes its amplitude from zero and stores its reduction term
};

struct Schedule {
    std::vector<Ins> ins;               // task instructions; operands are slots
    std::vector<uint32_t> task_first;   // tasks + 1 entries into ins
    std::vector<uint32_t> level_first;  // levels + 1 entries into tasks
    uint32_t cur_slots = 0;             // complex current slots per point
    uint32_t peak_live = 0;             // the most current slots live at one level (a floor for cur_slots)
    uint32_t amp_slots = 0;             // complex amplitude slots per point
    uint32_t terms = 0;                 // reduction terms per point (instead of amplitude slots)
    std::vector<uint32_t> loads;        // live-in currents: (global plane, slot, count) triples
    std::vector<uint32_t> amp_planes;   // per amplitude slot, its global amplitude plane
    std::vector<uint32_t> amp_slot_of;  // per global amplitude plane, its slot or ~0u
    uint32_t max_task_len = 0;
    std::vector<uint32_t> task_cost;    // per task, its algorithmic flops
    std::string why;                    // empty when the schedule exists
};

// The order in which a point's L lanes take a level's tasks: position j of a
// level goes to lane j % L, so each level is padded to whole rounds of L with ~0u (no task). The
// tasks of a level are assigned longest first to the least loaded lane.
void lane_order(const Schedule &s, uint32_t lanes, std::vector<uint32_t> &order, std::vector<uint32_t> &level_first);

// builds the schedule of a program; `forms` is the plan's momentum form count
bool build_schedule(const Program &p, uint32_t current_planes, uint32_t amplitude_planes, Schedule &out);

// For a run that only reduces its amplitudes (resolved from zero: offsets[outputs + 1], planes),
// when every amplitude gets exactly one closure row and feeds at most one of the reduction's
// terms: each closure row makes its amplitude from zero and stores its term (weight x |A|^2),
// and the points keep the terms (8 bytes each) instead of the amplitudes (16). False (the
// schedule unchanged) otherwise.
bool use_terms(Schedule &s, const uint32_t *offsets, const uint32_t *planes, uint32_t outputs, uint32_t amplitude_planes);

}  // namespace pacuda
