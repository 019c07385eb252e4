// Pipe.cpp -- the position bookkeeping of PipeBase (see Pipe.h).
#include "jengine/Pipe.h"

#include <algorithm>
#include <climits>

namespace JEngine {

namespace {
constexpr size_t kOpen = SIZE_MAX;  // end of a shot that is still being written
}

// Custom deleter of a token's shared info: the last copy going away releases
// the token in its pipe.
struct TokenReleaser {
    void operator()(PipeTokenInfo* info) const {
        if (info && info->owner) info->owner->Release(info);
        delete info;
    }
};

PipeBase::PipeBase(const std::string& name) : name(name) {}

PipeBase::~PipeBase() {
    std::unique_lock<std::mutex> lk(m);
    cv.wait(lk, [&] { return writes.empty() && reads.empty(); });
}

void PipeBase::SetConsumer(const std::string& who, size_t number, size_t size, size_t ov) {
    {
        std::lock_guard<std::mutex> lk(m);
        if (numReaders * readSize != 0) ThrowExceptionAndLog("consumer is already set.");
        if (number == 0) ThrowExceptionAndLog("number of reader can not be 0.");
        if (size == 0) ThrowExceptionAndLog("read size can not be 0.");
        if (ov >= size) ThrowExceptionAndLog("overlap must be smaller than the read size.");
        consumer = who;
        numReaders = number;
        readSize = size;
        overlap = ov;
    }
    MaybeAllocate();
    cv.notify_all();
}

void PipeBase::SetProducer(const std::string& who, size_t number, size_t size) {
    {
        std::lock_guard<std::mutex> lk(m);
        if (numWriters * writeSize != 0) ThrowExceptionAndLog("producer is already set.");
        if (number == 0) ThrowExceptionAndLog("number of writers can not be 0.");
        if (size == 0) ThrowExceptionAndLog("write size can not be 0.");
        producer = who;
        numWriters = number;
        writeSize = size;
    }
    MaybeAllocate();
    cv.notify_all();
}

void PipeBase::SetBufferSize(size_t size) {
    {
        std::lock_guard<std::mutex> lk(m);
        if (bufferSize != 0) ThrowExceptionAndLog("pipe size is already set.");
        bufferSize = size;
    }
    MaybeAllocate();
}

void PipeBase::MaybeAllocate() {
    std::lock_guard<std::mutex> lk(m);
    if (allocated || numReaders == 0 || numWriters == 0 || !hasTemplate) return;
    if (bufferSize == 0) bufferSize = numWriters * writeSize + numReaders * (readSize - overlap) + overlap;
    AllocateSlots(bufferSize);
    allocated = true;
    cv.notify_all();
}

size_t PipeBase::GetWriteDonePos() {
    std::lock_guard<std::mutex> lk(m);
    return writeDonePos;
}

size_t PipeBase::GetReadDonePos() {
    std::lock_guard<std::mutex> lk(m);
    return readDonePos;
}

void PipeBase::Close() {
    std::lock_guard<std::mutex> lk(m);
    closed = true;
    cv.notify_all();
}

bool PipeBase::Closed() {
    std::lock_guard<std::mutex> lk(m);
    return closed;
}

bool PipeBase::ReadReady(size_t& start, size_t& end) const {
    if (shots.empty() || !allocated) return false;
    const Shot& s = shots.front();
    start = std::max(s.start, readingPos > overlap ? readingPos - overlap : 0);
    end = std::min(start + readSize, s.end);
    return end > start && end <= std::min(writeDonePos, readDonePos + bufferSize);
}

size_t PipeBase::OldestNeeded() const {
    if (!reads.empty()) return reads.front().start;
    if (shots.empty()) return readingPos;
    return std::max(shots.front().start, readingPos > overlap ? readingPos - overlap : 0);
}

std::shared_ptr<PipeTokenInfo> PipeBase::AcquireWrite(size_t n, bool isShotEnd) {
    std::unique_lock<std::mutex> lk(m);
    if (allocated && n > bufferSize) ThrowExceptionAndLog("Pipe::GetWriteToken(): write size is larger than buffer size!");
    Timer t;
    while (!closed && !(allocated && writingPos + n <= OldestNeeded() + bufferSize)) {
        size_t a, b;
        if (allocated && writes.empty() && reads.empty() && !ReadReady(a, b)) {
            closed = true;
            cv.notify_all();
            ThrowExceptionAndLog("Pipe deadlock");
        }
        cv.wait(lk);
    }
    blockedTime += t.Toc();
    if (closed) ThrowExceptionAndLog("Pipe: trying to get write token when pipe is closed!");
    const bool shotStart = shots.empty() || shots.back().end != kOpen;
    if (shotStart) shots.push_back({writingPos, kOpen});
    auto* info = new PipeTokenInfo{this, writingPos, n, 0, shotStart, isShotEnd, false};
    writes.push_back({writingPos, n, false});
    writingPos += n;
    if (isShotEnd) {
        shots.back().end = writingPos;
        if (shots.back().end - shots.back().start < overlap + 1)
            ThrowExceptionAndLog("Shot size is smaller than or equal to overlap size.");
    }
    cv.notify_all();
    return std::shared_ptr<PipeTokenInfo>(info, TokenReleaser());
}

std::shared_ptr<PipeTokenInfo> PipeBase::AcquireRead() {
    std::unique_lock<std::mutex> lk(m);
    size_t start = 0, end = 0;
    while (!ReadReady(start, end)) {
        // Closed and nothing more can arrive: every write and read released
        // and what is left (if anything) cannot form a read.
        if (closed && writes.empty() && reads.empty()) throw PipeClosedAndEmptySignal();
        cv.wait(lk);
    }
    const Shot s = shots.front();
    const size_t ov = readingPos - start;
    auto* info = new PipeTokenInfo{this, start, end - start, ov, start == s.start, end == s.end, true};
    if (end == s.end) shots.pop_front();
    reads.push_back({start, end - start, false});
    readingPos += (end - start) - ov;
    cv.notify_all();
    return std::shared_ptr<PipeTokenInfo>(info, TokenReleaser());
}

void PipeBase::Release(PipeTokenInfo* info) {
    std::lock_guard<std::mutex> lk(m);
    auto& q = info->isRead ? reads : writes;
    for (auto& e : q)
        if (e.start == info->start && e.size == info->size && !e.done) {
            e.done = true;
            break;
        }
    while (!q.empty() && q.front().done) {
        if (info->isRead) readDonePos = q.front().start + q.front().size;
        else writeDonePos += q.front().size;
        q.pop_front();
    }
    cv.notify_all();
}

}  // namespace JEngine
