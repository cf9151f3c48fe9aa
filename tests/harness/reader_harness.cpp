// Test harness (CPU): the UMAMI library's .pacuda reader (pacuda_b200/umami/pacuda_reader.cpp)
// driven from Python: a text dump of what it read, compared with the Python reader's.
#include <inttypes.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>

#include "../../pacuda_b200/umami/pacuda_reader.h"

namespace {
void add(std::string &s, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void add(std::string &s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    s += buf;
}
template <class T> void list(std::string &s, const char *name, const std::vector<T> &v, const char *fmt) {
    s += name;
    for (const T &x : v) add(s, fmt, x);
    s += "\n";
}
}  // namespace

extern "C" {

// the dump of `path` into buf (NUL-terminated); its length, or -1 with the reader's reason in buf
int reader_dump(const char *path, char *buf, size_t cap) {
    pacuda::PacudaFile f;
    std::string why, s;
    if (!pacuda::read_pacuda(path, f, why)) {
        snprintf(buf, cap, "%s", why.c_str());
        return -1;
    }
    add(s, "file kernel %u batch %u shas %zu\n", f.kernel, f.batch, f.symjit_sha256.size());
    for (const auto &p : f.processes) {
        add(s, "process %s legs %u helicities %u alpha %s %.17g power %d factor %" PRId64 "/%" PRId64 "\n",
            p.key.c_str(), p.legs, p.helicities, p.alpha_s_name.c_str(), p.alpha_s, p.qcd_power, p.numerator,
            p.denominator);
        for (size_t k = 0; k < p.parameter_names.size(); k++)
            add(s, "parameter %s %.17g %.17g\n", p.parameter_names[k].c_str(), p.parameter_re[k], p.parameter_im[k]);
        list(s, "crossing", p.crossing_leg, " %u");
        list(s, "signs", p.crossing_sign, " %.17g");
        for (const auto &c : p.colours) {
            add(s, "colour %s tile %u words %zu key %016" PRIx64 " planes %u %u %u external %u outputs %u\n",
                c.id.c_str(), c.tile, c.words.size(), pacuda::program_key(c), c.current_planes, c.amplitude_planes,
                c.momentum_planes, c.external_count, c.outputs);
            s += "width";
            for (int k = 0; k < 8; k++) add(s, " %u", (unsigned)c.width[k]);
            s += "\n";
            list(s, "scale_re", c.scale_re, " %.17g");
            list(s, "factor_im", c.factor_im, " %.17g");
            list(s, "zero", c.zero, " %u");
            list(s, "download", c.download, " %u");
            list(s, "form_terms", c.form_terms, " %u");
            list(s, "term_slots", c.term_slots, " %u");
            list(s, "offsets", c.offsets, " %u");
            list(s, "live", c.live_helicity, " %u");
            list(s, "live_offsets", c.live_offsets, " %u");
            add(s, "reference %u %zu %zu\n", c.reference_points, c.reference_momenta.size(), c.reference_values.size());
        }
    }
    snprintf(buf, cap, "%s", s.c_str());
    return (int)s.size();
}
}
