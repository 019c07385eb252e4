// Pipe.h -- ring-buffer pipes between agents, with RAII read/write tokens.
//
// Behaviour of the reference's Pipeline/Pipe.h, Pipeline/PipeBase.cpp and
// Pipeline/Pipe{Read,Write}Token.h, restated for this library:
//  * positions grow without bound; element i lives in slot i % bufferSize;
//  * GetWriteToken(n, isShotEnd) blocks while the ring has no room for n
//    elements that every reader has released (PipeBase.cpp:147-201); a
//    writer that could never proceed (no token in flight, nothing readable)
//    closes the pipe and throws "Pipe deadlock" (PipeBase.cpp:203-221);
//  * writes are grouped into shots (a scan); a read never spans two shots;
//    reads of readSize elements overlap the previous read by overlapSize
//    (PipeBase.cpp:223-298);
//  * GetReadToken() blocks until a full read is written and throws
//    PipeClosedAndEmptySignal once the pipe is closed and drained;
//  * a token is released when its last copy dies; done positions advance in
//    token order (PipeBase.cpp:300-331);
//  * the default ring holds numWriters*writeSize + numReaders*(readSize -
//    overlap) + overlap elements (Pipeline/PipeImpl.h:84-89).
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "Common.h"

namespace JEngine {

struct PipeClosedAndEmptySignal {};

class PipeBase;

struct PipeTokenInfo {
    PipeBase* owner = nullptr;
    size_t start = 0, size = 0, overlap = 0;
    bool shotStart = false, shotEnd = false, isRead = false;
};

class PipeBase {
public:
    explicit PipeBase(const std::string& name);
    virtual ~PipeBase();
    PipeBase(const PipeBase&) = delete;
    PipeBase& operator=(const PipeBase&) = delete;

    void SetConsumer(const std::string& name, size_t number, size_t sizeIncludingOverlap, size_t overlapSize);
    void SetProducer(const std::string& name, size_t number, size_t size);
    void SetBufferSize(size_t size);
    std::vector<size_t> GetElementShape() const { return shape; }

    const std::string& GetName() const { return name; }
    const std::string& GetConsumer() const { return consumer; }
    const std::string& GetProducer() const { return producer; }
    size_t GetNumReaders() const { return numReaders; }
    size_t GetReadSize() const { return readSize; }
    size_t GetOverlapSize() const { return overlap; }
    size_t GetNumWriters() const { return numWriters; }
    size_t GetWriteSize() const { return writeSize; }
    size_t GetBufferSize() const { return bufferSize; }
    size_t GetWriteDonePos();
    size_t GetReadDonePos();

    void Close();
    bool Closed();
    double GetProducerBlockedTime() const { return blockedTime; }

protected:
    std::shared_ptr<PipeTokenInfo> AcquireWrite(size_t n, bool isShotEnd);
    std::shared_ptr<PipeTokenInfo> AcquireRead();
    void SetShape(const std::vector<size_t>& s) { shape = s; }
    virtual void AllocateSlots(size_t n) = 0;
    void MaybeAllocate();
    bool HasTemplate() const { return hasTemplate; }
    void MarkTemplate() { hasTemplate = true; }

private:
    friend struct TokenReleaser;
    void Release(PipeTokenInfo* info);
    bool ReadReady(size_t& start, size_t& end) const;  // under lock
    size_t OldestNeeded() const;                       // under lock

    struct Shot { size_t start, end; };
    struct Entry { size_t start, size; bool done; };

    std::string name, consumer, producer;
    std::vector<size_t> shape;
    size_t numWriters = 0, writeSize = 0, numReaders = 0, readSize = 0, overlap = 0, bufferSize = 0;
    bool allocated = false, hasTemplate = false, closed = false;

    std::mutex m;
    std::condition_variable cv;
    std::deque<Shot> shots;          // shots not yet fully read (end = SIZE_MAX while open)
    std::deque<Entry> writes, reads; // tokens in flight, in order
    size_t writingPos = 0, writeDonePos = 0, readingPos = 0, readDonePos = 0;
    double blockedTime = 0.0;
};

template <class T>
class PipeReadToken;
template <class T>
class PipeWriteToken;

template <class T>
class Pipe : public PipeBase {
public:
    typedef PipeWriteToken<T> WriteToken;
    typedef PipeReadToken<T> ReadToken;

    explicit Pipe(const std::string& name) : PipeBase(name) {}

    // Every slot is constructed as a copy of the template.
    void SetTemplate(T&& element, std::vector<size_t>&& dims) {
        if (HasTemplate()) ThrowExceptionAndLog("Pipe: buffer is already initialized.");
        buffers.clear();
        buffers.emplace_back(std::move(element));
        MarkTemplate();
        SetShape(dims);
        MaybeAllocate();
    }
    T GetTemplate() const {
        if (buffers.empty()) ThrowException("Pipe: pipe is not initialized.");
        return buffers[0];
    }

    WriteToken GetWriteToken(size_t n, bool isShotEnd) { return WriteToken(AcquireWrite(n, isShotEnd), this); }
    ReadToken GetReadToken() { return ReadToken(AcquireRead(), this); }

    T& Slot(size_t pos) { return buffers[pos % buffers.size()]; }
    // Slots allocated so far (0 until the pipe has its template, producer and consumer).
    size_t NumSlots() const { return buffers.size(); }

private:
    void AllocateSlots(size_t n) override { buffers.resize(n, buffers[0]); }
    std::vector<T> buffers;
};

template <class T>
class PipeReadToken {
public:
    PipeReadToken() = default;
    PipeReadToken(std::shared_ptr<PipeTokenInfo> info, Pipe<T>* pipe) : info(std::move(info)), pipe(pipe) {}
    PipeReadToken& operator=(const PipeReadToken& o) {
        if (info) ThrowException("ReadToken is already assigned.");
        info = o.info;
        pipe = o.pipe;
        return *this;
    }
    PipeReadToken(const PipeReadToken&) = default;
    bool Null() const { return !info; }
    size_t GetStartIndex() const { return info->start; }
    size_t GetSize() const { return info->size; }
    size_t GetOverlapSize() const { return info->overlap; }
    bool IsShotStart() const { return info->shotStart; }
    bool IsShotEnd() const { return info->shotEnd; }
    const T& GetBuffer(size_t i) const { return pipe->Slot(info->start + i); }
    T& GetMutableBuffer(size_t i) const { return pipe->Slot(info->start + i); }
    void Reset() { info.reset(); }

private:
    std::shared_ptr<PipeTokenInfo> info;
    Pipe<T>* pipe = nullptr;
};

template <class T>
class PipeWriteToken {
public:
    PipeWriteToken() = default;
    PipeWriteToken(std::shared_ptr<PipeTokenInfo> info, Pipe<T>* pipe) : info(std::move(info)), pipe(pipe) {}
    PipeWriteToken& operator=(const PipeWriteToken& o) {
        if (info) ThrowException("WriteToken is already assigned.");
        info = o.info;
        pipe = o.pipe;
        return *this;
    }
    PipeWriteToken(const PipeWriteToken&) = default;
    bool Null() const { return !info; }
    size_t GetStartIndex() const { return info->start; }
    size_t GetSize() const { return info->size; }
    bool IsShotStart() const { return info->shotStart; }
    bool IsShotEnd() const { return info->shotEnd; }
    T& GetBuffer(size_t i) const { return pipe->Slot(info->start + i); }
    void Reset() { info.reset(); }

private:
    std::shared_ptr<PipeTokenInfo> info;
    Pipe<T>* pipe = nullptr;
};

}  // namespace JEngine
