// The `.pacuda` v2 reader (pacuda_reader.h).
#include "pacuda_reader.h"

#include <stdio.h>
#include <string.h>

namespace pacuda {

namespace {

// A cursor over the file's bytes that turns bad, and stays bad, on any read past the end.
struct Cursor {
    const uint8_t *p, *end;
    bool bad = false;
    size_t left() const { return (size_t)(end - p); }
    bool take(void *out, size_t n) {
        if (bad || left() < n) {
            bad = true;
            return false;
        }
        if (out) memcpy(out, p, n);
        p += n;
        return true;
    }
    template <class T> T scalar() {
        T v{};
        take(&v, sizeof v);
        return v;
    }
    uint32_t u32() { return scalar<uint32_t>(); }
    template <class T> void array(std::vector<T> &v, size_t n) {
        if (bad || (n && n > left() / sizeof(T))) {
            bad = true;
            return;
        }
        v.resize(n);
        take(v.data(), n * sizeof(T));
    }
    std::string str() {
        uint32_t n = u32();
        if (bad || n > left()) {
            bad = true;
            return std::string();
        }
        std::string s((const char *)p, n);
        p += n;
        return s;
    }
    void runs(std::vector<uint32_t> &v) { array(v, 2 * (size_t)u32()); }
};

}  // namespace

bool parse_pacuda(const uint8_t *bytes, size_t size, PacudaFile &f, std::string &why) {
    Cursor r{bytes, bytes + size};
    char magic[8];
    if (!r.take(magic, 8) || memcmp(magic, "PACUDA\0\x01", 8) != 0 || r.u32() != 2) {
        why = "not a version-2 .pacuda file";
        return false;
    }
    f = PacudaFile();
    f.kernel = r.u32();
    f.batch = r.u32();
    uint32_t shas = r.u32();
    if (shas > r.left() / 64) r.bad = true;
    for (uint32_t k = 0; !r.bad && k < shas; k++) {
        char hex[64];
        r.take(hex, 64);
        f.symjit_sha256.emplace_back(hex, 64);
    }
    uint32_t processes = r.u32();
    for (uint32_t i = 0; !r.bad && i < processes; i++) {
        if (r.left() < 4) {
            r.bad = true;
            break;
        }
        f.processes.emplace_back();
        PacudaProcess &p = f.processes.back();
        p.key = r.str();
        p.legs = r.u32();
        p.helicities = r.u32();
        p.alpha_s_name = r.str();
        p.alpha_s = r.scalar<double>();
        p.qcd_power = r.scalar<int32_t>();
        uint32_t params = r.u32();
        if (params > r.left() / 20) r.bad = true;  // a name's length and two values at least
        for (uint32_t k = 0; !r.bad && k < params; k++) {
            p.parameter_names.push_back(r.str());
            p.parameter_re.push_back(r.scalar<double>());
            p.parameter_im.push_back(r.scalar<double>());
        }
        p.numerator = r.scalar<int64_t>();
        p.denominator = r.scalar<int64_t>();
        uint32_t crossing = r.u32();
        if (crossing && crossing != p.legs) r.bad = true;
        for (uint32_t l = 0; !r.bad && l < crossing; l++) {
            p.crossing_leg.push_back(r.u32());
            p.crossing_sign.push_back(r.scalar<double>());
            if (p.crossing_leg.back() >= p.legs) r.bad = true;
        }
        uint32_t colours = r.u32();
        for (uint32_t j = 0; !r.bad && j < colours; j++) {
            if (r.left() < 4) {
                r.bad = true;
                break;
            }
            p.colours.emplace_back();
            PacudaColour &c = p.colours.back();
            c.id = r.str();
            c.tile = r.u32();
            r.array(c.words, r.u32());
            r.take(c.width, 8);
            c.current_planes = r.u32();
            c.amplitude_planes = r.u32();
            c.momentum_planes = r.u32();
            uint32_t n = r.u32();
            r.array(c.scale_re, n);
            r.array(c.scale_im, n);
            n = r.u32();
            r.array(c.factor_re, n);
            r.array(c.factor_im, n);
            r.runs(c.zero);
            r.runs(c.download);
            c.external_count = r.u32();
            r.runs(c.form_terms);
            n = r.u32();
            r.array(c.term_slots, n);
            r.array(c.term_coefficients, n);
            c.outputs = r.u32();
            if (c.outputs == UINT32_MAX) r.bad = true;
            if (!r.bad) r.array(c.offsets, (size_t)c.outputs + 1);
            uint32_t terms = r.bad || c.offsets.empty() ? 0 : c.offsets[c.outputs];
            r.array(c.planes, terms);
            r.array(c.weights, terms);
            c.reference_points = r.u32();
            r.array(c.reference_momenta, (size_t)c.reference_points * p.legs * 4);
            r.array(c.reference_values, (size_t)c.reference_points * p.helicities);
            if (r.bad) break;
            if (c.outputs != p.helicities || c.external_count != p.legs || c.tile == 0 || c.offsets[0] != 0) {
                r.bad = true;
                break;
            }
            for (uint32_t h = 0; h < c.outputs; h++)
                if (c.offsets[h] > c.offsets[h + 1]) r.bad = true;
            for (uint32_t h = 0; !r.bad && h < c.outputs; h++)
                if (c.offsets[h + 1] > c.offsets[h]) {
                    c.live_offsets.push_back(c.offsets[h]);
                    c.live_helicity.push_back(h);
                }
            c.live_offsets.push_back(c.offsets[c.outputs]);
        }
    }
    if (!r.bad && r.p != r.end) {
        why = "bytes after the last process";
        return false;
    }
    if (r.bad) {
        why = "a malformed .pacuda file";
        return false;
    }
    return true;
}

bool read_pacuda(const char *path, PacudaFile &out, std::string &why) {
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        why = std::string(path) + ": cannot open";
        return false;
    }
    std::vector<uint8_t> bytes;
    uint8_t chunk[1 << 16];
    size_t n;
    while ((n = fread(chunk, 1, sizeof chunk, fp)) > 0) bytes.insert(bytes.end(), chunk, chunk + n);
    bool err = ferror(fp) != 0;
    fclose(fp);
    if (err) {
        why = std::string(path) + ": cannot read";
        return false;
    }
    if (!parse_pacuda(bytes.data(), bytes.size(), out, why)) {
        why = std::string(path) + ": " + why;
        return false;
    }
    return true;
}

uint64_t program_key(const PacudaColour &c) {
    // the reference's starting value (one digit short of FNV's published offset basis), kept so
    // that a program's key here equals the reference library's
    uint64_t h = 1469598103934665603ull;
    for (int k = 0; k < 8; k++) h = (h ^ c.width[k]) * 1099511628211ull;
    const uint8_t *b = (const uint8_t *)c.words.data();
    for (size_t k = 0; k < c.words.size() * 8; k++) h = (h ^ b[k]) * 1099511628211ull;
    return h ? h : 1;
}

}  // namespace pacuda
