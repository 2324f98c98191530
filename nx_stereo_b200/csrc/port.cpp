// nxs_port: the reference's stereo_match Port (native/stereo_match/src/main.rs)
// served by this library on a B200, so NxStereo.Matcher and NativeSegment,
// unmodified, run their segments on the GPU when the Matcher's :path option
// names this binary. The protocol is port_records.h's; records are framed as
// {:packet, 4} (a big-endian length before each record).
//
// Three threads, as stereo_match has: one reads and parses requests, one
// hands them to the library (a configure waits for the device; a run is
// enqueued with nxs_run_async and does not), and one writes the replies in
// the order of the requests, waiting for each run's outputs on the device.
// Runs of one segment are computed in the order sent (nxs_run_async), so up
// to kInFlight pairs overlap on the device while replies keep their order.
//
// `nxs_port [--threads N] [--device D]`: N is accepted for stereo_match's
// sake and ignored (the GPU computes); D picks the CUDA device (0). The CUDA
// context opens on the first configure: without a device, every configure
// is refused with the reason. stdout carries records only (fd 1 is pointed
// at stderr, so a library printing cannot corrupt the framing).
#include <unistd.h>

#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "port_records.h"

namespace {

constexpr size_t kInFlight = 4;  // requests enqueued on the device at once

FILE *records_out = nullptr;  // the real stdout
std::mutex write_lock;

bool write_record(const std::vector<uint8_t> &record) {
    std::lock_guard<std::mutex> g(write_lock);
    const uint32_t n = (uint32_t)record.size();
    const uint8_t length[4] = {(uint8_t)(n >> 24), (uint8_t)(n >> 16), (uint8_t)(n >> 8),
                               (uint8_t)n};
    return fwrite(length, 1, 4, records_out) == 4 &&
           fwrite(record.data(), 1, record.size(), records_out) == record.size() &&
           fflush(records_out) == 0;
}

bool read_exact(uint8_t *buffer, size_t n) {
    size_t got = 0;
    while (got < n) {
        const ssize_t r = read(0, buffer + got, n - got);
        if (r <= 0) return false;  // end of input (the Port closed) or an error
        got += (size_t)r;
    }
    return true;
}

// One record, or false at the end of the input.
bool read_record(std::vector<uint8_t> *record) {
    uint8_t length[4];
    if (!read_exact(length, 4)) return false;
    const uint32_t n = (uint32_t)length[0] << 24 | (uint32_t)length[1] << 16 |
                       (uint32_t)length[2] << 8 | length[3];
    record->resize(n);
    return n == 0 || read_exact(record->data(), n);
}

// What the writer replies with, in request order.
struct Reply {
    std::vector<uint8_t> record;      // ready to write, or
    nxs_request *request = nullptr;   // a run whose outputs the writer waits for
};

template <typename T>
class Queue {  // a bounded FIFO between two threads
  public:
    explicit Queue(size_t capacity) : capacity_(capacity) {}
    void push(T item) {
        std::unique_lock<std::mutex> l(m_);
        not_full_.wait(l, [&] { return items_.size() < capacity_; });
        items_.push_back(std::move(item));
        not_empty_.notify_one();
    }
    void close() {
        std::lock_guard<std::mutex> l(m_);
        closed_ = true;
        not_empty_.notify_all();
    }
    bool pop(T *item) {
        std::unique_lock<std::mutex> l(m_);
        not_empty_.wait(l, [&] { return !items_.empty() || closed_; });
        if (items_.empty()) return false;
        *item = std::move(items_.front());
        items_.pop_front();
        not_full_.notify_one();
        return true;
    }

  private:
    size_t capacity_;
    std::deque<T> items_;
    bool closed_ = false;
    std::mutex m_;
    std::condition_variable not_empty_, not_full_;
};

struct Parsed {
    std::vector<uint8_t> bytes;  // the record, which the request's entries point into
    std::unique_ptr<nxs_port::Request> request;
    std::string refusal;         // why it does not parse
};

}  // namespace

int main(int argc, char **argv) {
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if ((a == "--threads" || a == "--device") && i + 1 < argc) {
            const int v = std::atoi(argv[++i]);
            if (v < (a == "--threads" ? 1 : 0)) {
                fprintf(stderr, "%s takes a %s integer\n", a.c_str(),
                        a == "--threads" ? "positive" : "non-negative");
                return 2;
            }
            if (a == "--device") device = v;
        } else {
            fprintf(stderr, "usage: nxs_port [--threads N] [--device D]\n");
            return 2;
        }
    }
    const int saved = dup(1);
    if (saved < 0 || dup2(2, 1) < 0 || !(records_out = fdopen(saved, "wb"))) return 1;
    write_record(nxs_port::log_record(0, std::string(nxs_version()) + " on CUDA device " +
                                             std::to_string(device)));

    Queue<Parsed> parsed(2);
    Queue<Reply> replies(kInFlight);
    std::thread reader([&] {
        for (;;) {
            Parsed p;
            if (!read_record(&p.bytes)) break;
            p.request.reset(new nxs_port::Request());
            if (!nxs_port::parse(p.bytes.data(), p.bytes.size(), p.request.get(), &p.refusal))
                p.request.reset();
            parsed.push(std::move(p));
        }
        parsed.close();
    });
    std::thread writer([&] {
        Reply r;
        bool open = true;
        while (replies.pop(&r)) {
            if (r.request) {
                char error[512] = "";
                if (nxs_request_wait(r.request, -1, error, sizeof error) != NXS_OK ||
                    !nxs_port::outputs_record(r.request, &r.record))
                    r.record = nxs_port::refused_record(error[0] ? error : "the run failed");
                nxs_request_free(r.request);
            }
            if (open && !write_record(r.record)) open = false;  // the Port closed: drain
        }
    });

    nxs_context *context = nullptr;
    std::string no_context;
    Parsed p;
    while (parsed.pop(&p)) {
        Reply reply;
        if (!p.request) {
            reply.record = nxs_port::refused_record(p.refusal);
            replies.push(std::move(reply));
            continue;
        }
        const nxs_port::Request &q = *p.request;
        char error[512] = "";
        if (q.kind == nxs_port::kRelease) {
            if (context) nxs_release(context, q.segment);
            continue;  // not replied to
        }
        if (!context && no_context.empty() &&
            nxs_create(device, &context, error, sizeof error) != NXS_OK)
            no_context = std::string("no CUDA device: ") + error;
        if (!context) {
            reply.record = nxs_port::refused_record(no_context);
        } else if (q.kind == nxs_port::kConfigure) {
            if (nxs_configure(context, q.segment, &q.geometry, (uint32_t)q.members.size(),
                              q.members.data(), error, sizeof error) == NXS_OK) {
                reply.record = {nxs_port::kTagConfigured};
            } else {
                nxs_release(context, q.segment);  // a refused configuration leaves none
                reply.record = nxs_port::refused_record(error);
            }
        } else {  // run: enqueued now, its outputs waited for by the writer
            nxs_request *request = nullptr;
            const nxs_status s =
                nxs_run_async(context, q.segment, (uint32_t)q.params.size(), q.params.data(),
                              (uint32_t)q.entries.size(), q.entries.data(), nullptr, nullptr, 0,
                              &request, error, sizeof error);
            if (s == NXS_OK) reply.request = request;
            else if (s == NXS_NO_SEGMENT)
                reply.record = nxs_port::refused_record("segment " + std::to_string(q.segment) +
                                                        " is not configured");
            else reply.record = nxs_port::refused_record(error);
        }
        replies.push(std::move(reply));
    }
    replies.close();
    writer.join();
    reader.join();
    if (context) nxs_destroy(context);
    return 0;
}
