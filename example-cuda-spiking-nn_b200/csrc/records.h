// records.h -- the text files the reference's monitors write, and a writer thread for them.
//
// Monitor::record (cpp_src/monitors/spike_recorder.cpp:40-60, voltage_recorder.cpp:54-78,
// weight_recorder.cpp:25-51) downloads a ring buffer and writes it as text on the host thread
// that steps the simulation.  Here the download stays on that thread (the ring must be copied
// out before the next steps overwrite it) and the formatting and file writes go to one writer
// thread per simulation, so the GPU keeps stepping while text is written.  The bytes written are
// the reference's, quirks included:
//  * spike rows: "<label>, <id> <id> ... \n" per ring slot, labels first_step + slot where
//    first_step = clock_step - interval, so slot 0 (which holds step clock_step) is labelled
//    clock_step - interval; nothing is written while clock_step < interval;
//  * voltage files: one file per ring slot, named by inserting "_step<clock_step - interval +
//    slot + 1>" before ".txt" (32-bit unsigned arithmetic, as the reference computes it, so the
//    record at clock step 0 wraps around), each "neuron_id, voltage\n" then one line per selected
//    neuron in selection order;
//  * weight files: at clock steps that are multiples of 100,000, "pre_neuron_id, post_neuron_id,
//    weight\n" then every (pre, post) pair including zeros.
// Floats are printed as std::ostream prints a float by default (printf "%g" of its double value).
#pragma once

#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <deque>
#include <fstream>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace bsnn {
namespace rec {

inline void put_u32(std::string& s, uint32_t v) {
    char b[16];
    const int n = std::snprintf(b, sizeof b, "%u", v);
    s.append(b, static_cast<size_t>(n));
}

inline void put_float(std::string& s, float v) {
    char b[48];
    const int n = std::snprintf(b, sizeof b, "%g", static_cast<double>(v));
    s.append(b, static_cast<size_t>(n));
}

// The reference's "_step<N>" file name: inserted before the last ".txt" of `path`.
inline std::string step_path(const std::string& path, uint32_t step) {
    std::string f = path;
    f.insert(f.rfind(".txt"), "_step" + std::to_string(step));
    return f;
}

// Spike rows of one record: `bits` is the ring, time-major [interval][words] (bit b of word w =
// neuron 32 w + b of the group).
inline void spike_rows(std::string& out, const uint32_t* bits, uint32_t words, uint32_t n_neurons, uint32_t interval,
                       uint32_t clock_step) {
    const uint32_t first_step = clock_step - interval;
    for (uint32_t slot = 0; slot < interval; ++slot) {
        put_u32(out, first_step + slot);
        out += ", ";
        const uint32_t* row = bits + static_cast<size_t>(slot) * words;
        for (uint32_t w = 0; w < words; ++w) {
            uint32_t m = row[w];
            while (m) {
                const uint32_t b = static_cast<uint32_t>(__builtin_ctz(m));
                m &= m - 1u;
                const uint32_t id = 32u * w + b;
                if (id >= n_neurons) break;
                put_u32(out, id);
                out += ' ';
            }
        }
        out += '\n';
    }
}

// One voltage file: `vh` is the ring [interval][n_cols]; `col[k]` is the ring column of the k-th
// selected neuron `sel[k]`.
inline void voltage_file(std::string& out, const std::vector<uint32_t>& sel, const std::vector<uint32_t>& col,
                         const float* vh, uint32_t n_cols, uint32_t slot) {
    out += "neuron_id, voltage\n";
    for (size_t k = 0; k < sel.size(); ++k) {
        put_u32(out, sel[k]);
        out += ", ";
        put_float(out, vh[static_cast<size_t>(slot) * n_cols + col[k]]);
        out += '\n';
    }
}

// One weight file from a row-major [n_pre][ld] matrix.
inline void weight_file(std::string& out, const float* w, uint32_t n_pre, uint32_t n_post, uint32_t ld) {
    out += "pre_neuron_id, post_neuron_id, weight\n";
    for (uint32_t i = 0; i < n_pre; ++i)
        for (uint32_t q = 0; q < n_post; ++q) {
            put_u32(out, i);
            out += ", ";
            put_u32(out, q);
            out += ", ";
            put_float(out, w[static_cast<size_t>(i) * ld + q]);
            out += '\n';
        }
}

// Writes `data` to a new file at `path` (truncating); a file that cannot be opened is skipped,
// as the reference skips output when its stream is not good().
inline void write_file(const std::string& path, const std::string& data) {
    std::ofstream f(path, std::ios::out | std::ios::trunc | std::ios::binary);
    if (!f.good()) return;
    f.write(data.data(), static_cast<std::streamsize>(data.size()));
}

// One background thread running queued jobs in order.
class Writer {
public:
    Writer() : th_([this] { loop(); }) {}
    ~Writer() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        th_.join();
    }
    void push(std::function<void()> job) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(job));
            ++pending_;
        }
        cv_.notify_all();
    }
    // Blocks until every queued job has run.
    void drain() {
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

private:
    void loop() {
        for (;;) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                job = std::move(q_.front());
                q_.pop_front();
            }
            job();
            {
                std::lock_guard<std::mutex> lk(mu_);
                --pending_;
            }
            done_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<std::function<void()>> q_;
    size_t pending_ = 0;
    bool stop_ = false;
    std::thread th_;
};

}  // namespace rec
}  // namespace bsnn
