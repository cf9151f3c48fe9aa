// The `.pacuda` plan file, version 2, read into memory (C++).
//
// The format is the reference converter's (convert/src/format.rs:1-29), as the reference's UMAMI
// library reads it (umami/umami_pacuda.c:149-279): little endian, sequential, no padding; arrays
// follow their counts, strings their byte lengths (u32, no NUL), run lists their number of
// (first, count) pairs. Every count is checked against the bytes left before anything is
// allocated, and the file must end after its last process.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace pacuda {

struct PacudaColour {
    std::string id;
    uint32_t tile = 0;
    std::vector<uint64_t> words;
    uint8_t width[8] = {0};
    uint32_t current_planes = 0, amplitude_planes = 0, momentum_planes = 0;
    std::vector<double> scale_re, scale_im, factor_re, factor_im;
    std::vector<uint32_t> zero, download;  // runs: (first, count) pairs
    uint32_t external_count = 0;
    std::vector<uint32_t> form_terms;       // (first term, term count) per form
    std::vector<uint32_t> term_slots;
    std::vector<double> term_coefficients;
    uint32_t outputs = 0;                   // one per helicity
    std::vector<uint32_t> offsets, planes;  // the resolved reduction
    std::vector<double> weights;
    // the outputs that reduce any plane, in order, and their offsets (live + 1 entries)
    std::vector<uint32_t> live_helicity, live_offsets;
    uint32_t reference_points = 0;
    std::vector<double> reference_momenta, reference_values;
};

struct PacudaProcess {
    std::string key;
    uint32_t legs = 0, helicities = 0;
    std::string alpha_s_name;
    double alpha_s = 0.0;
    int32_t qcd_power = 0;
    std::vector<std::string> parameter_names;
    std::vector<double> parameter_re, parameter_im;
    int64_t numerator = 1, denominator = 1;  // the process-group factor
    std::vector<uint32_t> crossing_leg;      // empty: identity
    std::vector<double> crossing_sign;
    std::vector<PacudaColour> colours;
};

struct PacudaFile {
    uint32_t kernel = 0, batch = 0;
    std::vector<std::string> symjit_sha256;
    std::vector<PacudaProcess> processes;
};

// Reads `path`; false (with the reason in `why`) when it cannot be read or is malformed.
bool read_pacuda(const char *path, PacudaFile &out, std::string &why);
// The same from bytes in memory.
bool parse_pacuda(const uint8_t *bytes, size_t size, PacudaFile &out, std::string &why);

// The runner's cache key of a colour's program: 64-bit FNV-1a over its eight widths and then its
// words' bytes, never 0 (umami/umami_pacuda.c:300-307: the same program gets the same key in
// every library, so the runner compiles it once).
uint64_t program_key(const PacudaColour &c);

}  // namespace pacuda
