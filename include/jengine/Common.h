// Common.h -- utilities shared by the pipeline runtime and the agents:
// exceptions, element typedefs, a closable blocking queue, a counting
// semaphore, a timer and a thread-safe logger.
//
// Same names and behaviour as the reference's Common/ (Common/Exception.h:
// 12-41, Common/TypeDefs.h:7-11, Common/SyncQueue.h, Common/Semaphore.h,
// Common/Timer.h, Common/GLog.h), written for this library.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <exception>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

namespace JEngine {

typedef std::vector<float> FloatVec;
typedef std::vector<unsigned short> UINT16Vec;
typedef std::vector<signed short> INT16Vec;
typedef std::vector<unsigned char> ByteVec;

// Global log sink.  Defaults to stderr; tests install their own.
void GLogWrite(const std::string& msg);
void SetGLogSink(std::function<void(const std::string&)> sink);
#define GLog(msg) ::JEngine::GLogWrite(msg)

class Exception : public std::exception {
public:
    Exception(const std::string& file, size_t line, const std::string& msg, bool log);
    const char* what() const noexcept override { return message.c_str(); }
    std::string What() const { return message; }

private:
    std::string message;
};

#define ThrowExceptionAndLog(msg) throw ::JEngine::Exception(__FILE__, __LINE__, msg, true)
#define ThrowException(msg) throw ::JEngine::Exception(__FILE__, __LINE__, msg, false)

struct SyncQueueClosedAndEmptySignal {};

// Blocking FIFO with an optional capacity; Pop throws
// SyncQueueClosedAndEmptySignal once the queue is closed and drained.
template <class T>
class SyncQueue {
public:
    explicit SyncQueue(size_t capacity = 0) : cap(capacity) {}
    void Push(T v) {
        std::unique_lock<std::mutex> lk(m);
        notFull.wait(lk, [&] { return closed || cap == 0 || q.size() < cap; });
        if (closed) ThrowException("SyncQueue: push after close");
        q.push_back(std::move(v));
        notEmpty.notify_one();
    }
    T Pop() {
        std::unique_lock<std::mutex> lk(m);
        notEmpty.wait(lk, [&] { return closed || !q.empty(); });
        if (q.empty()) throw SyncQueueClosedAndEmptySignal();
        T v = std::move(q.front());
        q.pop_front();
        notFull.notify_one();
        return v;
    }
    void Close() {
        std::lock_guard<std::mutex> lk(m);
        closed = true;
        notEmpty.notify_all();
        notFull.notify_all();
    }
    size_t Size() {
        std::lock_guard<std::mutex> lk(m);
        return q.size();
    }

private:
    std::mutex m;
    std::condition_variable notEmpty, notFull;
    std::deque<T> q;
    size_t cap;
    bool closed = false;
};

// Counting semaphore: Wait(n) blocks until n signals accumulated, consumes them.
class Semaphore {
public:
    explicit Semaphore(size_t initial = 0) : count(initial) {}
    void Signal(size_t n = 1) {
        std::lock_guard<std::mutex> lk(m);
        count += n;
        cv.notify_all();
    }
    void Wait(size_t n = 1) {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return count >= n; });
        count -= n;
    }

private:
    std::mutex m;
    std::condition_variable cv;
    size_t count;
};

class Timer {
public:
    Timer() : t0(std::chrono::steady_clock::now()) {}
    void Tic() { t0 = std::chrono::steady_clock::now(); }
    double Toc() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

private:
    std::chrono::steady_clock::time_point t0;
};

}  // namespace JEngine
