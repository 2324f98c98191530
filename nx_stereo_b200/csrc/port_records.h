// The records of the reference's native Port protocol
// (native/stereo_match/src/protocol.rs:1-23, framing.rs:1-44), decoded into
// and encoded from this library's C ABI: the codec behind nxs_port (a drop-in
// for the stereo_match binary) and the NIF. A request is one record: its kind
// (1 configure, 2 run, 3 release), a u32 segment id, then
//   configure: width, height, frame_width, frame_height (u16), the member
//              count (u8), each member's kind (a name) and options: a count
//              (u8), then each option's name and f64 value;
//   run:       the member count (u8), each member's live inputs: a count (u8),
//              each input's name, value count (u16) and f32 values; then the
//              entries: a count (u8) and each a tensor;
//   release:   nothing more.
// A name is its length (u8) and bytes; a tensor its name, type (u8: 0 u8,
// 1 u16, 2 f32, 3 s32), rank (u8), dimensions (u32) and row-major elements.
// Scalars are little-endian. Replies: 7 (configured), 8 then each member's
// time (u8 count, u32 us) and the output tensors (u8 count), 9 and a reason.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nx_stereo_b200.h"

namespace nxs_port {

constexpr uint8_t kConfigure = 1, kRun = 2, kRelease = 3;
constexpr uint8_t kTagLog = 2, kTagConfigured = 7, kTagOutputs = 8, kTagRefused = 9;

// A decoded request. The C ABI views (members, params, entries) point into
// the request's own storage and, for entry elements, into the record bytes,
// which must outlive them.
struct Request {
    uint8_t kind = 0;
    uint32_t segment = 0;
    nxs_geometry geometry{};
    // configure
    std::vector<std::string> kinds;
    std::vector<std::vector<std::string>> option_names;
    std::vector<std::vector<nxs_setting>> options;
    std::vector<nxs_member> members;
    // run
    std::vector<std::vector<std::string>> input_names;
    std::vector<std::vector<std::vector<float>>> input_values;
    std::vector<std::vector<nxs_param>> inputs;
    std::vector<nxs_member_params> params;
    std::vector<std::string> entry_names;
    std::vector<nxs_tensor> entries;
};

class Reader {
  public:
    Reader(const uint8_t *data, size_t size) : at_(data), end_(data + size) {}
    bool take(size_t n, const uint8_t **out, std::string *why) {
        if (n > (size_t)(end_ - at_)) {
            *why = "the request ends " + std::to_string(n - (size_t)(end_ - at_)) +
                   " bytes early";
            return false;
        }
        *out = at_;
        at_ += n;
        return true;
    }
    template <typename T>
    bool scalar(T *out, std::string *why) {
        const uint8_t *p;
        if (!take(sizeof(T), &p, why)) return false;
        T v = 0;
        for (size_t i = 0; i < sizeof(T); ++i) v |= (T)p[i] << (8 * i);  // little-endian
        *out = v;
        return true;
    }
    bool f64(double *out, std::string *why) {
        uint64_t bits;
        if (!scalar(&bits, why)) return false;
        std::memcpy(out, &bits, 8);
        return true;
    }
    bool name(std::string *out, std::string *why) {
        uint8_t n;
        const uint8_t *p;
        if (!scalar(&n, why) || !take(n, &p, why)) return false;
        out->assign(reinterpret_cast<const char *>(p), n);
        return true;
    }
    size_t left() const { return (size_t)(end_ - at_); }

  private:
    const uint8_t *at_, *end_;
};

inline size_t element_bytes(uint8_t type) {
    return type == NXS_U8 ? 1 : type == NXS_U16 ? 2 : (type == NXS_F32 || type == NXS_S32) ? 4 : 0;
}

// Parses one request record (protocol.rs:98-158, with its refusals: a record
// that ends early, bytes after it, an unknown kind, an unknown tensor type).
inline bool parse(const uint8_t *data, size_t size, Request *r, std::string *why) {
    Reader in(data, size);
    if (!in.scalar(&r->kind, why) || !in.scalar(&r->segment, why)) return false;
    if (r->kind == kConfigure) {
        uint16_t w, h, fw, fh;
        uint8_t count;
        if (!in.scalar(&w, why) || !in.scalar(&h, why) || !in.scalar(&fw, why) ||
            !in.scalar(&fh, why) || !in.scalar(&count, why))
            return false;
        r->geometry = nxs_geometry{w, h, fw, fh};
        r->kinds.resize(count);
        r->option_names.resize(count);
        r->options.resize(count);
        for (uint8_t m = 0; m < count; ++m) {
            uint8_t n;
            if (!in.name(&r->kinds[m], why) || !in.scalar(&n, why)) return false;
            r->option_names[m].resize(n);
            r->options[m].resize(n);
            for (uint8_t k = 0; k < n; ++k)
                if (!in.name(&r->option_names[m][k], why) || !in.f64(&r->options[m][k].value, why))
                    return false;
        }
        for (uint8_t m = 0; m < count; ++m) {
            for (size_t k = 0; k < r->options[m].size(); ++k)
                r->options[m][k].name = r->option_names[m][k].c_str();
            r->members.push_back(nxs_member{r->kinds[m].c_str(), (uint32_t)r->options[m].size(),
                                            r->options[m].data()});
        }
    } else if (r->kind == kRun) {
        uint8_t count;
        if (!in.scalar(&count, why)) return false;
        r->input_names.resize(count);
        r->input_values.resize(count);
        r->inputs.resize(count);
        for (uint8_t m = 0; m < count; ++m) {
            uint8_t n;
            if (!in.scalar(&n, why)) return false;
            r->input_names[m].resize(n);
            r->input_values[m].resize(n);
            for (uint8_t k = 0; k < n; ++k) {
                uint16_t values;
                const uint8_t *p;
                if (!in.name(&r->input_names[m][k], why) || !in.scalar(&values, why) ||
                    !in.take(4 * (size_t)values, &p, why))
                    return false;
                r->input_values[m][k].resize(values);
                std::memcpy(r->input_values[m][k].data(), p, 4 * (size_t)values);
            }
        }
        for (uint8_t m = 0; m < count; ++m) {
            for (size_t k = 0; k < r->input_names[m].size(); ++k)
                r->inputs[m].push_back(nxs_param{r->input_names[m][k].c_str(),
                                                 (uint32_t)r->input_values[m][k].size(),
                                                 r->input_values[m][k].data()});
            r->params.push_back(nxs_member_params{(uint32_t)r->inputs[m].size(),
                                                  r->inputs[m].data()});
        }
        uint8_t n_entries;
        if (!in.scalar(&n_entries, why)) return false;
        r->entry_names.resize(n_entries);
        for (uint8_t e = 0; e < n_entries; ++e) {
            nxs_tensor t{};
            uint8_t type, rank;
            if (!in.name(&r->entry_names[e], why) || !in.scalar(&type, why) ||
                !in.scalar(&rank, why))
                return false;
            if (!element_bytes(type)) {
                *why = "unknown tensor type " + std::to_string(type);
                return false;
            }
            if (rank > 4) {
                *why = "a tensor of rank " + std::to_string(rank);
                return false;
            }
            size_t elements = 1;
            for (uint8_t d = 0; d < rank; ++d) {
                if (!in.scalar(&t.dims[d], why)) return false;
                elements *= t.dims[d];
            }
            const uint8_t *p;
            if (!in.take(elements * element_bytes(type), &p, why)) return false;
            t.type = type;
            t.rank = rank;
            t.data = p;
            t.bytes = elements * element_bytes(type);
            r->entries.push_back(t);
        }
        for (uint8_t e = 0; e < n_entries; ++e) r->entries[e].name = r->entry_names[e].c_str();
    } else if (r->kind != kRelease) {
        *why = "unknown request kind " + std::to_string(r->kind);
        return false;
    }
    if (in.left()) {
        *why = std::to_string(in.left()) + " bytes follow the request";
        return false;
    }
    return true;
}

inline void put_u32(std::vector<uint8_t> *out, uint32_t v) {
    for (int i = 0; i < 4; ++i) out->push_back((uint8_t)(v >> (8 * i)));
}

// The outputs reply of a finished request (protocol.rs:160-199): tag 8, each
// member's time, then the tensors the members filled.
inline bool outputs_record(nxs_request *request, std::vector<uint8_t> *out) {
    uint32_t n_times = 0, n_outputs = 0;
    const uint32_t *times = nullptr;
    const nxs_tensor *outputs = nullptr;
    if (nxs_request_times(request, &n_times, &times) != NXS_OK ||
        nxs_request_outputs(request, &n_outputs, &outputs) != NXS_OK)
        return false;
    out->clear();
    out->push_back(kTagOutputs);
    out->push_back((uint8_t)n_times);
    for (uint32_t i = 0; i < n_times; ++i) put_u32(out, times[i]);
    out->push_back((uint8_t)n_outputs);
    for (uint32_t i = 0; i < n_outputs; ++i) {
        const nxs_tensor &t = outputs[i];
        const size_t name = std::strlen(t.name);
        out->push_back((uint8_t)name);
        out->insert(out->end(), t.name, t.name + name);
        out->push_back((uint8_t)t.type);
        out->push_back((uint8_t)t.rank);
        for (uint32_t d = 0; d < t.rank; ++d) put_u32(out, t.dims[d]);
        const uint8_t *bytes = static_cast<const uint8_t *>(t.data);
        out->insert(out->end(), bytes, bytes + t.bytes);
    }
    return true;
}

// The refusal reply (protocol.rs:150-153): tag 9 and the reason.
inline std::vector<uint8_t> refused_record(const std::string &reason) {
    std::vector<uint8_t> out{kTagRefused};
    out.insert(out.end(), reason.begin(), reason.end());
    return out;
}

// A log record (framing.rs): tag 2, the level (0 info, 1 warning, 2 error), the text.
inline std::vector<uint8_t> log_record(uint8_t level, const std::string &text) {
    std::vector<uint8_t> out{kTagLog, level};
    out.insert(out.end(), text.begin(), text.end());
    return out;
}

}  // namespace nxs_port
