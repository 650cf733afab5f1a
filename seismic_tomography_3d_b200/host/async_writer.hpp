// Background file writer for the plug-in classes (header only, so that it compiles inside
// the reference's tree as well as here).
//
// The reference writes every per-shot first-arrival file, every recovered model and every
// illumination volume with a blocking std::ofstream in the middle of the iteration
// (block_FIM.cpp:260, least_squares.cpp:290/567).  Here the caller hands the data over and
// goes on: the bytes are copied, queued, and written by one background thread with the same
// layout, the same path and the same "was succesfully written" line as the reference's
// write_binary_float.  Files are written in the order they were queued.
//
// drain() waits until every queued file is on disk.  A failed write (the file could not be
// opened or written) is kept and thrown as std::invalid_argument -- the reference's
// exception type -- by the next write_floats() or drain() on any thread; the process-wide
// instance drains itself at exit.
#ifndef TOMO_B200_ASYNC_WRITER_HPP
#define TOMO_B200_ASYNC_WRITER_HPP

#include <condition_variable>
#include <cstddef>
#include <deque>
#include <exception>
#include <fstream>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace tomo_io {

class AsyncWriter {
public:
    // The process-wide writer the plug-ins share.
    static AsyncWriter &instance()
    {
        static AsyncWriter w;
        return w;
    }

    AsyncWriter() : worker_([this] { run(); }) {}
    AsyncWriter(const AsyncWriter &) = delete;
    AsyncWriter &operator=(const AsyncWriter &) = delete;

    ~AsyncWriter()
    {
        try {
            drain();
        } catch (const std::exception &e) {
            std::cerr << e.what() << std::endl;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        work_.notify_all();
        worker_.join();
    }

    // Copies n floats and queues them for `path`; returns without waiting for the disk.
    void write_floats(const std::string &path, const float *data, size_t n)
    {
        Job j{path, std::vector<float>(data, data + n)};
        std::unique_lock<std::mutex> lk(m_);
        rethrow_locked();
        q_.push_back(std::move(j));
        lk.unlock();
        work_.notify_one();
    }

    // Waits until every queued file is written; throws the first failure seen since the
    // last throw.
    void drain()
    {
        std::unique_lock<std::mutex> lk(m_);
        idle_.wait(lk, [this] { return q_.empty() && !busy_; });
        rethrow_locked();
    }

private:
    struct Job {
        std::string path;
        std::vector<float> data;
    };

    void rethrow_locked()
    {
        if (err_) {
            std::exception_ptr e = err_;
            err_ = nullptr;
            std::rethrow_exception(e);
        }
    }

    void run()
    {
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            work_.wait(lk, [this] { return stop_ || !q_.empty(); });
            if (q_.empty()) return;  // stop requested and nothing left
            Job j = std::move(q_.front());
            q_.pop_front();
            busy_ = true;
            lk.unlock();
            std::exception_ptr e;
            try {
                std::ofstream f(j.path, std::ios::out | std::ios::binary);
                if (!f.is_open()) throw std::invalid_argument("Error: file could not be opened! (" + j.path + ")");
                f.write(reinterpret_cast<const char *>(j.data.data()),
                        (std::streamsize)(j.data.size() * sizeof(float)));
                f.close();
                if (!f) throw std::invalid_argument("Error: file could not be written! (" + j.path + ")");
                std::cout << "Binary file " + j.path + " was succesfully written." << std::endl;
            } catch (...) {
                e = std::current_exception();
            }
            lk.lock();
            if (e && !err_) err_ = e;
            busy_ = false;
            if (q_.empty()) idle_.notify_all();
        }
    }

    std::mutex m_;
    std::condition_variable work_, idle_;
    std::deque<Job> q_;
    bool busy_ = false, stop_ = false;
    std::exception_ptr err_;
    std::thread worker_;  // last: started once every other member exists
};

}  // namespace tomo_io

#endif
