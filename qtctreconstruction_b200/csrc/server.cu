// server.cu — the serving loop (ctb_server_*) and its admission allocator
// (ctb_arena_*). No counterpart in the reference, whose controller runs one
// reconstruction per call on a worker thread (CtReconstructionController.cpp:
// 1096-1146).
//
// Threads and streams:
//   scheduler   admits queued requests in arrival order while their device
//               footprint fits the budget (one arena block per request: angle
//               table, filtered rows, and unless the request is device-resident
//               its sinograms and volume), then packs requests whose data is on
//               the device into batches on the compute stream: one filter launch
//               per convolution length and one backprojection launch per tile
//               shape over all (request, slice group, tile) items,
//               at most two batches queued at a time so the GPU never waits for
//               the host between batches.
//   uploaders   fill a request's angle table and copy its host sinograms on
//               their own stream: directly from page-locked memory, else
//               through a pinned double buffer.
//   downloaders copy finished volumes back the same way and release the
//               request's arena block, which lets the scheduler admit the next
//               requests.
// A batch's completion is signalled by a host callback on the compute stream
// (cudaLaunchHostFunc), which only touches host state. Requests that arrive
// while others run join the next batch: continuous batching.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

#include "api_util.h"

using namespace ctb;
using Clock = std::chrono::steady_clock;

// ------------------------------------------------------------------ arena
struct ctb_arena {
    size_t capacity = 0;
    size_t used = 0;
    size_t peak = 0;
    std::map<size_t, size_t> free_ranges;         // offset -> bytes
    std::unordered_map<size_t, size_t> held;      // offset -> bytes
};

namespace {

constexpr size_t kUnit = 256;
size_t round_unit(size_t b) { return (b + kUnit - 1) / kUnit * kUnit; }

void arena_init(ctb_arena* a, size_t capacity) {
    a->capacity = capacity / kUnit * kUnit;
    a->used = a->peak = 0;
    a->free_ranges.clear();
    a->held.clear();
    if (a->capacity) a->free_ranges.emplace(0, a->capacity);
}

bool arena_alloc(ctb_arena* a, size_t bytes, size_t* off) {
    bytes = round_unit(std::max<size_t>(bytes, 1));
    for (auto it = a->free_ranges.begin(); it != a->free_ranges.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t o = it->first, rest = it->second - bytes;
        a->free_ranges.erase(it);
        if (rest) a->free_ranges.emplace(o + bytes, rest);
        a->held.emplace(o, bytes);
        a->used += bytes;
        a->peak = std::max(a->peak, a->used);
        *off = o;
        return true;
    }
    return false;
}

bool arena_free(ctb_arena* a, size_t off) {
    auto h = a->held.find(off);
    if (h == a->held.end()) return false;
    size_t bytes = h->second;
    a->held.erase(h);
    a->used -= bytes;
    auto next = a->free_ranges.lower_bound(off);
    if (next != a->free_ranges.end() && off + bytes == next->first) {
        bytes += next->second;
        next = a->free_ranges.erase(next);
    }
    if (next != a->free_ranges.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += bytes;
            return true;
        }
    }
    a->free_ranges.emplace(off, bytes);
    return true;
}

size_t arena_largest(const ctb_arena* a) {
    size_t m = 0;
    for (const auto& kv : a->free_ranges) m = std::max(m, kv.second);
    return m;
}

// ------------------------------------------------------------ requests
enum State { kPending, kAdmitted, kReady, kComputing, kDownloading, kFinal };

struct SReq {
    uint64_t id = 0;
    uint64_t seq = 0;
    ctb_request r{};
    std::vector<float> angles;
    State state = kPending;
    ctb_status status = CTB_ERR_BUSY;
    bool cancel = false;
    bool has_block = false;
    size_t off = 0;
    size_t bytes = 0;
    size_t sino_bytes = 0, out_bytes = 0, trig_off = 0, filt_off = 0, sino_off = 0, out_off = 0;
    const float* d_sino = nullptr;
    float4* d_filt = nullptr;
    void* d_trig = nullptr;
    float* d_out = nullptr;
    PadGeom g;
    FiltLayout fl;
    const float2* Hc = nullptr;
    const float2* tw = nullptr;
    Clock::time_point t_submit, t_done;
    double updates = 0.0;
    int bypassed = 0;
};

// A copy thread's stream and pinned double buffer.
struct Stager {
    cudaStream_t stream = nullptr;
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    size_t half = 0;
};

constexpr int kMaxInflightBatches = 2;
constexpr int kErrSlots = 8;
constexpr int kMaxBypass = 16;  // times the oldest request may be overtaken by smaller ones

}  // namespace

struct ctb_server;

namespace {
struct BatchRec {
    ctb_server* s = nullptr;
    std::vector<SReq*> reqs;
    int slot = 0;
};
}  // namespace

struct ctb_server {
    ctb_server_config cfg{};
    char* d_base = nullptr;
    ctb_arena arena;
    cudaStream_t compute = nullptr;
    cudaStream_t table_stream = nullptr;
    int sms = 0;
    unsigned* d_err = nullptr;  // [0] error word of bounded waits, [1] backprojection item counter
    unsigned* h_err = nullptr;  // pinned, one word per batch slot
    std::vector<Stager> up_st, down_st;

    std::mutex mu;
    std::condition_variable cv_sched, cv_up, cv_down, cv_done;
    std::deque<SReq*> pending, upq, downq, ready;
    std::unordered_map<uint64_t, std::unique_ptr<SReq>> reqs;
    std::mutex tables_mu;  // guards filters / twiddles (never held with mu)
    std::map<std::pair<int, int>, DevBuf> filters;
    std::map<int, DevBuf> twiddles;
    bool kick = false;     // something changed that may let a queued request in
    int inflight = 0;
    uint64_t batch_seq = 0;
    int workers_busy = 0;
    bool stop = false;
    uint64_t next_id = 1;
    std::thread sched;
    std::vector<std::thread> up, down;

    uint64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0;
    uint64_t batches = 0, batched = 0;
    std::vector<double> lat_ms;
    bool have_first = false;
    Clock::time_point t_first, t_last;
    double updates_done = 0.0;
};

namespace {

// -------------------------------------------------------------- footprint
void plan_request(SReq* q) {
    const ctb_request& r = q->r;
    q->g = pad_geometry(r.bins);
    q->fl = filt_layout(q->g.sq, r.output_size);
    size_t off = 0;
    q->trig_off = off;
    off += round_unit((sizeof(double2) + sizeof(float2)) * static_cast<size_t>(r.num_angles));
    q->filt_off = off;
    off += round_unit(sizeof(float4) * static_cast<size_t>((r.depth + 3) / 4) * r.num_angles * q->fl.pitch);
    q->sino_bytes = sizeof(float) * static_cast<size_t>(r.depth) * r.num_angles * r.bins;
    q->out_bytes = sizeof(float) * static_cast<size_t>(r.depth) * r.output_size * r.output_size;
    if (!(r.flags & CTB_REQ_DEVICE)) {
        q->sino_off = off;
        off += round_unit(q->sino_bytes);
        q->out_off = off;
        off += round_unit(q->out_bytes);
    }
    q->bytes = off;
    q->updates = static_cast<double>(r.output_size) * r.output_size * r.depth * r.num_angles;
}

// Mark a request final and release its arena block (mu held).
void finalize(ctb_server* s, SReq* q, ctb_status st) {
    if (q->state == kFinal) return;
    if (q->has_block) {
        arena_free(&s->arena, q->off);
        q->has_block = false;
    }
    q->state = kFinal;
    q->status = st;
    q->t_done = Clock::now();
    if (st == CTB_OK) {
        ++s->completed;
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count());
        s->t_last = q->t_done;
        s->updates_done += q->updates;
    } else if (st == CTB_ERR_CANCELLED) {
        ++s->cancelled;
    } else {
        ++s->failed;
    }
    s->kick = true;
    s->cv_done.notify_all();
    s->cv_sched.notify_all();
}

// Convolution spectrum and twiddles for a request (server cache; called at
// submission with tables_mu held and mu not held: no CUDA call ever runs under
// mu, which the batch callbacks take).
ctb_status request_tables(ctb_server* s, SReq* q) {
    const int Lc = q->g.Lc;
    auto key = std::make_pair(q->r.bins, q->r.filter);
    auto it = s->filters.find(key);
    if (it == s->filters.end()) {
        const std::vector<float2> Hc = filter_table(q->g, q->r.filter);
        DevBuf b;
        if (cudaMalloc(&b.ptr, sizeof(float2) * Hc.size()) != cudaSuccess) return CTB_ERR_OOM;
        b.bytes = sizeof(float2) * Hc.size();
        if (cudaMemcpyAsync(b.ptr, Hc.data(), b.bytes, cudaMemcpyHostToDevice, s->table_stream) != cudaSuccess ||
            cudaStreamSynchronize(s->table_stream) != cudaSuccess) {
            cudaFree(b.ptr);
            return CTB_ERR_CUDA;
        }
        it = s->filters.emplace(key, b).first;
    }
    auto jt = s->twiddles.find(Lc);
    if (jt == s->twiddles.end()) {
        const std::vector<float2> tw = fft_twiddle_table(Lc);
        DevBuf b;
        if (cudaMalloc(&b.ptr, sizeof(float2) * tw.size()) != cudaSuccess) return CTB_ERR_OOM;
        b.bytes = sizeof(float2) * tw.size();
        if (cudaMemcpyAsync(b.ptr, tw.data(), b.bytes, cudaMemcpyHostToDevice, s->table_stream) != cudaSuccess ||
            cudaStreamSynchronize(s->table_stream) != cudaSuccess) {
            cudaFree(b.ptr);
            return CTB_ERR_CUDA;
        }
        jt = s->twiddles.emplace(Lc, b).first;
    }
    q->Hc = static_cast<const float2*>(it->second.ptr);
    q->tw = static_cast<const float2*>(jt->second.ptr);
    return CTB_OK;
}

// Admit queued requests in arrival order while they fit (mu held). A request
// that does not fit may be overtaken by smaller ones, the oldest such request
// at most kMaxBypass times.
void admit(ctb_server* s) {
    SReq* blocked = nullptr;
    for (auto it = s->pending.begin(); it != s->pending.end();) {
        SReq* q = *it;
        size_t off = 0;
        if (!arena_alloc(&s->arena, q->bytes, &off)) {
            if (!blocked) {
                blocked = q;
                if (q->bypassed >= kMaxBypass) return;
            }
            ++it;
            continue;
        }
        if (blocked) ++blocked->bypassed;
        it = s->pending.erase(it);
        q->off = off;
        q->has_block = true;
        char* base = s->d_base + off;
        q->d_trig = base + q->trig_off;
        q->d_filt = reinterpret_cast<float4*>(base + q->filt_off);
        if (q->r.flags & CTB_REQ_DEVICE) {
            q->d_sino = q->r.sino;
            q->d_out = q->r.out;
        } else {
            q->d_sino = reinterpret_cast<const float*>(base + q->sino_off);
            q->d_out = reinterpret_cast<float*>(base + q->out_off);
        }
        q->state = kAdmitted;
        s->upq.push_back(q);
        s->cv_up.notify_one();
    }
}

void CUDART_CB batch_done(void* p);

// Launch one batch on the compute stream (mu not held).
ctb_status launch_batch(ctb_server* s, const std::vector<SReq*>& reqs, int slot) {
    const int n = static_cast<int>(reqs.size());
    // filter launches per convolution length
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a]->g.Lc < reqs[b]->g.Lc; });
    for (int k = 0; k < n;) {
        FiltBatch f;
        f.Lc = reqs[order[k]]->g.Lc;
        f.tw = reqs[order[k]]->tw;
        while (k < n && f.njobs < kMaxJobs && reqs[order[k]]->g.Lc == f.Lc) {
            const SReq* q = reqs[order[k]];
            const float scale = 3.14159265358979323846f / (2.0f * static_cast<float>(q->r.num_angles));
            FiltJob J = make_filt_job(q->d_sino, q->r.depth, q->r.num_angles, q->g, q->fl, q->Hc, nullptr,
                                      CTB_DENORM_NONE, scale, q->d_filt);
            J.first = f.total;
            f.total += static_cast<long long>(J.na) * ((J.nz + 1) / 2);
            f.job[f.njobs++] = J;
            ++k;
        }
        if (launch_filter_batch(f, s->compute) != cudaSuccess) return CTB_ERR_CUDA;
    }
    // one backprojection launch per tile shape (the default shape of each
    // request, a function of its size), one CTA per (request, slice group,
    // tile) item, most angles first
    std::vector<int> var(n);
    for (int k = 0; k < n; ++k) var[k] = bp_default_variant(reqs[k]->r.output_size, reqs[k]->r.depth, s->sms);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return var[a] != var[b] ? var[a] < var[b] : reqs[a]->r.num_angles > reqs[b]->r.num_angles;
    });
    for (int k = 0; k < n;) {
        BpBatch bp;
        const int v = var[order[k]];
        while (k < n && bp.njobs < kMaxJobs && var[order[k]] == v) {
            const SReq* q = reqs[order[k]];
            Trig trig;
            trig.cs = static_cast<const double2*>(q->d_trig);
            trig.csf = reinterpret_cast<const float2*>(static_cast<const double2*>(q->d_trig) + q->r.num_angles);
            BpJob J = make_bp_job(q->d_filt, q->r.depth, q->r.num_angles, q->fl, q->r.output_size, trig, nullptr,
                                  CTB_DENORM_NONE, q->d_out, v);
            J.first = bp.total;
            bp.total += static_cast<long long>(J.tiles) * ((J.nz + 3) / 4);
            bp.job[bp.njobs++] = J;
            ++k;
        }
        if (launch_backproject_batch(bp, v, s->d_err + 1, s->d_err, s->compute) != cudaSuccess) return CTB_ERR_CUDA;
    }
    if (cudaMemcpyAsync(s->h_err + slot, s->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->compute) !=
            cudaSuccess ||
        cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), s->compute) != cudaSuccess)
        return CTB_ERR_CUDA;
    return CTB_OK;
}

void scheduler(ctb_server* s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_sched.wait_for(lk, std::chrono::milliseconds(50), [&] {
            return s->stop || s->kick || (!s->ready.empty() && s->inflight < kMaxInflightBatches);
        });
        s->kick = false;
        if (s->stop) {
            while (!s->ready.empty()) {
                finalize(s, s->ready.front(), CTB_ERR_CANCELLED);
                s->ready.pop_front();
            }
            break;
        }
        admit(s);
        while (!s->ready.empty() && s->inflight < kMaxInflightBatches) {
            std::vector<SReq*> batch;
            while (!s->ready.empty() && static_cast<int>(batch.size()) < s->cfg.max_batch) {
                SReq* q = s->ready.front();
                s->ready.pop_front();
                if (q->cancel) {
                    finalize(s, q, CTB_ERR_CANCELLED);
                    continue;
                }
                q->state = kComputing;
                batch.push_back(q);
            }
            if (batch.empty()) break;
            auto* rec = new BatchRec();
            rec->s = s;
            rec->reqs = batch;
            rec->slot = static_cast<int>(s->batch_seq++ % kErrSlots);
            ++s->inflight;
            ++s->batches;
            s->batched += batch.size();
            lk.unlock();
            ctb_status st = launch_batch(s, batch, rec->slot);
            if (st == CTB_OK && cudaLaunchHostFunc(s->compute, batch_done, rec) != cudaSuccess) st = CTB_ERR_CUDA;
            lk.lock();
            if (st != CTB_OK) {
                for (SReq* q : batch) finalize(s, q, st);
                --s->inflight;
                delete rec;
            }
        }
    }
}

// Host callback after a batch finished on the compute stream: no CUDA calls.
void CUDART_CB batch_done(void* p) {
    BatchRec* rec = static_cast<BatchRec*>(p);
    ctb_server* s = rec->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const unsigned err = s->h_err[rec->slot];
        for (SReq* q : rec->reqs) {
            if (err) {
                finalize(s, q, CTB_ERR_TIMEOUT);
            } else if (q->cancel) {
                finalize(s, q, CTB_ERR_CANCELLED);
            } else if (q->r.flags & CTB_REQ_DEVICE) {
                finalize(s, q, CTB_OK);
            } else {
                q->state = kDownloading;
                s->downq.push_back(q);
            }
        }
        --s->inflight;
        s->cv_down.notify_all();
        s->cv_sched.notify_all();
    }
    delete rec;
}

// Angle table: double2 cs via the device sincospi kernel from degrees staged in
// the (not yet used) filtered-row region, then the reference's float cos/sin.
bool upload_trig(SReq* q, Stager& st) {
    const int na = q->r.num_angles;
    std::vector<float2> csf(na);
    for (int a = 0; a < na; ++a) {
        const float th = q->angles[a] * 3.14159265358979323846f / 180.0f;
        csf[a] = make_float2(std::cos(th), std::sin(th));
    }
    float* d_deg = reinterpret_cast<float*>(q->d_filt);
    double2* cs = static_cast<double2*>(q->d_trig);
    return cudaMemcpyAsync(d_deg, q->angles.data(), sizeof(float) * na, cudaMemcpyHostToDevice, st.stream) ==
               cudaSuccess &&
           cudaMemcpyAsync(cs + na, csf.data(), sizeof(float2) * na, cudaMemcpyHostToDevice, st.stream) ==
               cudaSuccess &&
           launch_trig(d_deg, na, cs, st.stream) == cudaSuccess &&
           cudaStreamSynchronize(st.stream) == cudaSuccess;
}

// A host buffer the copy engines can read or write directly (page-locked by
// cudaHostAlloc or cudaHostRegister); pageable memory goes through the pinned
// double buffers.
bool page_locked(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host -> device: straight from page-locked memory, else through the pinned
// double buffer (chunk k is copied into buffer k & 1 once that buffer's
// previous transfer has finished).
bool staged_h2d(Stager& st, void* dst, const void* src, size_t bytes) {
    if (page_locked(src))
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st.stream) == cudaSuccess &&
               cudaStreamSynchronize(st.stream) == cudaSuccess;
    const char* s8 = static_cast<const char*>(src);
    char* d8 = static_cast<char*>(dst);
    int k = 0;
    for (size_t off = 0; off < bytes; off += st.half, k ^= 1) {
        const size_t len = std::min(st.half, bytes - off);
        if (cudaEventSynchronize(st.ev[k]) != cudaSuccess) return false;
        std::memcpy(st.pin[k], s8 + off, len);
        if (cudaMemcpyAsync(d8 + off, st.pin[k], len, cudaMemcpyHostToDevice, st.stream) != cudaSuccess ||
            cudaEventRecord(st.ev[k], st.stream) != cudaSuccess)
            return false;
    }
    return cudaStreamSynchronize(st.stream) == cudaSuccess;
}

// Device -> host: straight into page-locked memory, else chunk k lands in
// buffer k & 1 while chunk k - 1 is copied out.
bool staged_d2h(Stager& st, void* dst, const void* src, size_t bytes) {
    if (page_locked(dst))
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st.stream) == cudaSuccess &&
               cudaStreamSynchronize(st.stream) == cudaSuccess;
    const char* s8 = static_cast<const char*>(src);
    char* d8 = static_cast<char*>(dst);
    size_t prev_off = 0, prev_len = 0;
    int k = 0;
    for (size_t off = 0; off < bytes; off += st.half, k ^= 1) {
        const size_t len = std::min(st.half, bytes - off);
        if (cudaMemcpyAsync(st.pin[k], s8 + off, len, cudaMemcpyDeviceToHost, st.stream) != cudaSuccess ||
            cudaEventRecord(st.ev[k], st.stream) != cudaSuccess)
            return false;
        if (prev_len) {
            if (cudaEventSynchronize(st.ev[k ^ 1]) != cudaSuccess) return false;
            std::memcpy(d8 + prev_off, st.pin[k ^ 1], prev_len);
        }
        prev_off = off;
        prev_len = len;
    }
    if (prev_len) {
        if (cudaEventSynchronize(st.ev[k ^ 1]) != cudaSuccess) return false;
        std::memcpy(d8 + prev_off, st.pin[k ^ 1], prev_len);
    }
    return true;
}

void uploader(ctb_server* s, int idx) {
    cudaSetDevice(s->cfg.device);
    Stager& st = s->up_st[idx];
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_up.wait(lk, [&] { return s->stop || !s->upq.empty(); });
        if (s->upq.empty()) {
            if (s->stop) break;
            continue;
        }
        SReq* q = s->upq.front();
        s->upq.pop_front();
        if (q->cancel || s->stop) {
            finalize(s, q, CTB_ERR_CANCELLED);
            continue;
        }
        ++s->workers_busy;
        lk.unlock();
        bool ok = !(s->cfg.fault_every > 0 && q->seq % static_cast<uint64_t>(s->cfg.fault_every) == 0);
        if (ok) ok = upload_trig(q, st);
        if (ok && !(q->r.flags & CTB_REQ_DEVICE))
            ok = staged_h2d(st, const_cast<float*>(q->d_sino), q->r.sino, q->sino_bytes);
        if (!ok) cudaGetLastError();
        lk.lock();
        --s->workers_busy;
        if (!ok) {
            finalize(s, q, CTB_ERR_CUDA);
        } else if (q->cancel) {
            finalize(s, q, CTB_ERR_CANCELLED);
        } else {
            q->state = kReady;
            s->ready.push_back(q);
            s->cv_sched.notify_all();
        }
    }
}

void downloader(ctb_server* s, int idx) {
    cudaSetDevice(s->cfg.device);
    Stager& st = s->down_st[idx];
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_down.wait(lk, [&] { return (s->stop && s->inflight == 0) || !s->downq.empty(); });
        if (s->downq.empty()) {
            if (s->stop && s->inflight == 0) break;
            continue;
        }
        SReq* q = s->downq.front();
        s->downq.pop_front();
        if (q->cancel) {
            finalize(s, q, CTB_ERR_CANCELLED);
            continue;
        }
        ++s->workers_busy;
        lk.unlock();
        const bool ok = staged_d2h(st, q->r.out, q->d_out, q->out_bytes);
        if (!ok) cudaGetLastError();
        lk.lock();
        --s->workers_busy;
        finalize(s, q, ok ? CTB_OK : CTB_ERR_CUDA);
    }
}

bool make_stager(Stager& st, size_t bytes) {
    st.half = std::max<size_t>(bytes / 2, 1 << 20);
    if (cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    for (int k = 0; k < 2; ++k) {
        if (cudaHostAlloc(&st.pin[k], st.half, cudaHostAllocDefault) != cudaSuccess) return false;
        if (cudaEventCreateWithFlags(&st.ev[k], cudaEventDisableTiming) != cudaSuccess) return false;
    }
    return true;
}

void free_stager(Stager& st) {
    for (int k = 0; k < 2; ++k) {
        if (st.pin[k]) cudaFreeHost(st.pin[k]);
        if (st.ev[k]) cudaEventDestroy(st.ev[k]);
    }
    if (st.stream) cudaStreamDestroy(st.stream);
}

void free_server(ctb_server* s) {
    for (auto& st : s->up_st) free_stager(st);
    for (auto& st : s->down_st) free_stager(st);
    for (auto& kv : s->filters) cudaFree(kv.second.ptr);
    for (auto& kv : s->twiddles) cudaFree(kv.second.ptr);
    if (s->d_base) cudaFree(s->d_base);
    if (s->d_err) cudaFree(s->d_err);
    if (s->h_err) cudaFreeHost(s->h_err);
    if (s->compute) cudaStreamDestroy(s->compute);
    if (s->table_stream) cudaStreamDestroy(s->table_stream);
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    const size_t k = std::min(v.size() - 1, static_cast<size_t>(std::ceil(p * v.size())) - (p > 0 ? 1 : 0));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ arena
ctb_status ctb_arena_create(size_t capacity, ctb_arena** out) {
    if (!out) return CTB_ERR_INVALID;
    *out = nullptr;
    if (capacity < kUnit) return CTB_ERR_INVALID;
    auto* a = new ctb_arena();
    arena_init(a, capacity);
    *out = a;
    return CTB_OK;
}

ctb_status ctb_arena_alloc(ctb_arena* a, size_t bytes, size_t* offset) {
    if (!a || !offset) return CTB_ERR_INVALID;
    return arena_alloc(a, bytes, offset) ? CTB_OK : CTB_ERR_OOM;
}

ctb_status ctb_arena_free(ctb_arena* a, size_t offset) {
    if (!a) return CTB_ERR_INVALID;
    return arena_free(a, offset) ? CTB_OK : CTB_ERR_NOT_FOUND;
}

ctb_status ctb_arena_stats(const ctb_arena* a, size_t* used, size_t* peak, size_t* largest_free) {
    if (!a) return CTB_ERR_INVALID;
    if (used) *used = a->used;
    if (peak) *peak = a->peak;
    if (largest_free) *largest_free = arena_largest(a);
    return CTB_OK;
}

void ctb_arena_destroy(ctb_arena* a) { delete a; }

// ----------------------------------------------------------------- server
ctb_status ctb_server_create(const ctb_server_config* config, ctb_server** out) {
    if (!out) return CTB_ERR_INVALID;
    *out = nullptr;
    ctb_server_config cfg{};
    if (config) cfg = *config;
    if (cfg.max_batch <= 0 || cfg.max_batch > kMaxJobs) cfg.max_batch = kMaxJobs;
    if (cfg.copy_threads <= 0) cfg.copy_threads = 4;
    if (cfg.copy_threads > 32) cfg.copy_threads = 32;
    if (cfg.staging_bytes == 0) cfg.staging_bytes = size_t(64) << 20;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || cfg.device < 0 || cfg.device >= count) {
        cudaGetLastError();
        return CTB_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, cfg.device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return CTB_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(cfg.device) != cudaSuccess) return CTB_ERR_CUDA;
    if (cfg.memory_budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        cfg.memory_budget = std::min<size_t>(size_t(120) << 30, static_cast<size_t>(0.85 * fr));
    }
    auto* s = new ctb_server();
    s->cfg = cfg;
    s->sms = prop.multiProcessorCount;
    bool ok = cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->table_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&s->d_err, 2 * sizeof(unsigned)) == cudaSuccess &&
              cudaMemset(s->d_err, 0, 2 * sizeof(unsigned)) == cudaSuccess &&
              cudaHostAlloc(&s->h_err, kErrSlots * sizeof(unsigned), cudaHostAllocDefault) == cudaSuccess;
    if (ok && cudaMalloc(&s->d_base, cfg.memory_budget) != cudaSuccess) {
        cudaGetLastError();
        free_server(s);
        delete s;
        return CTB_ERR_OOM;
    }
    s->up_st.resize(cfg.copy_threads);
    s->down_st.resize(cfg.copy_threads);
    for (int i = 0; ok && i < cfg.copy_threads; ++i)
        ok = make_stager(s->up_st[i], cfg.staging_bytes) && make_stager(s->down_st[i], cfg.staging_bytes);
    if (!ok) {
        cudaGetLastError();
        free_server(s);
        delete s;
        return CTB_ERR_CUDA;
    }
    arena_init(&s->arena, cfg.memory_budget);
    s->sched = std::thread(scheduler, s);
    for (int i = 0; i < cfg.copy_threads; ++i) {
        s->up.emplace_back(uploader, s, i);
        s->down.emplace_back(downloader, s, i);
    }
    *out = s;
    return CTB_OK;
}

ctb_status ctb_server_submit(ctb_server* s, const ctb_request* req, uint64_t* id) {
    if (!s || !req || !id) return CTB_ERR_INVALID;
    const ctb_request& r = *req;
    if (!r.sino || !r.out || r.depth <= 0 || r.num_angles <= 0 || r.num_angles > kMaxAngles || r.bins <= 0 ||
        r.output_size <= 0 || r.filter < 0 || r.filter > CTB_FILTER_BARTLETT || (r.flags & ~CTB_REQ_DEVICE))
        return CTB_ERR_INVALID;
    if (pad_geometry(r.bins).Lc > kMaxFft) return CTB_ERR_UNSUPPORTED;
    auto q = std::make_unique<SReq>();
    q->r = r;
    if (r.angles_deg)
        q->angles.assign(r.angles_deg, r.angles_deg + r.num_angles);
    else
        q->angles = uniform_angles(r.num_angles);
    q->r.angles_deg = nullptr;
    plan_request(q.get());
    if (q->bytes <= s->arena.capacity) {  // capacity is fixed at creation
        std::lock_guard<std::mutex> tl(s->tables_mu);
        const ctb_status st = request_tables(s, q.get());
        if (st != CTB_OK) return st;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return CTB_ERR_CANCELLED;
    if (q->bytes > s->arena.capacity) {
        ++s->rejected;
        return CTB_ERR_OOM;
    }
    q->id = s->next_id++;
    q->seq = ++s->submitted;
    q->t_submit = Clock::now();
    if (!s->have_first) {
        s->have_first = true;
        s->t_first = q->t_submit;
    }
    SReq* raw = q.get();
    s->reqs.emplace(raw->id, std::move(q));
    s->pending.push_back(raw);
    *id = raw->id;
    s->kick = true;
    s->cv_sched.notify_all();
    return CTB_OK;
}

ctb_status ctb_server_poll(ctb_server* s, uint64_t id) {
    if (!s) return CTB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CTB_ERR_NOT_FOUND;
    return it->second->state == kFinal ? it->second->status : CTB_ERR_BUSY;
}

ctb_status ctb_server_wait(ctb_server* s, uint64_t id, double timeout_ms) {
    if (!s) return CTB_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CTB_ERR_NOT_FOUND;
    SReq* q = it->second.get();
    auto done = [&] { return q->state == kFinal; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done))
        return CTB_ERR_BUSY;
    return q->status;
}

ctb_status ctb_server_cancel(ctb_server* s, uint64_t id) {
    if (!s) return CTB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CTB_ERR_NOT_FOUND;
    SReq* q = it->second.get();
    if (q->state == kFinal) return CTB_OK;
    q->cancel = true;
    if (q->state == kPending) {
        s->pending.erase(std::find(s->pending.begin(), s->pending.end(), q));
        finalize(s, q, CTB_ERR_CANCELLED);
    }
    return CTB_OK;
}

ctb_status ctb_server_release(ctb_server* s, uint64_t id) {
    if (!s) return CTB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CTB_ERR_NOT_FOUND;
    if (it->second->state != kFinal) return CTB_ERR_BUSY;
    s->reqs.erase(it);
    return CTB_OK;
}

ctb_status ctb_server_get_stats(ctb_server* s, ctb_server_stats* out) {
    if (!s || !out) return CTB_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    ctb_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.failed = s->failed;
    st.cancelled = s->cancelled;
    st.rejected = s->rejected;
    st.batches = s->batches;
    st.mean_batch = s->batches ? static_cast<double>(s->batched) / s->batches : 0.0;
    st.p50_ms = percentile(s->lat_ms, 0.50);
    st.p99_ms = percentile(s->lat_ms, 0.99);
    st.max_ms = s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end());
    if (s->completed && s->have_first) {
        const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        if (span > 0) {
            st.volumes_per_s = s->completed / span;
            st.updates_per_s = s->updates_done / span;
        }
    }
    st.memory_budget = s->arena.capacity;
    st.memory_peak = s->arena.peak;
    *out = st;
    return CTB_OK;
}

void ctb_server_destroy(ctb_server* s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->stop = true;
        while (!s->pending.empty()) {
            finalize(s, s->pending.front(), CTB_ERR_CANCELLED);
            s->pending.pop_front();
        }
        for (auto& kv : s->reqs)
            if (kv.second->state != kFinal) kv.second->cancel = true;
        s->cv_sched.notify_all();
        s->cv_up.notify_all();
        s->cv_down.notify_all();
    }
    if (s->sched.joinable()) s->sched.join();
    for (auto& t : s->up)
        if (t.joinable()) t.join();
    cudaSetDevice(s->cfg.device);
    cudaStreamSynchronize(s->compute);  // runs the remaining batch callbacks
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv_down.notify_all();
    }
    for (auto& t : s->down)
        if (t.joinable()) t.join();
    {
        // requests uploaded after the scheduler stopped never reached a batch
        std::lock_guard<std::mutex> lk(s->mu);
        for (SReq* q : s->ready) finalize(s, q, CTB_ERR_CANCELLED);
        s->ready.clear();
        for (SReq* q : s->upq) finalize(s, q, CTB_ERR_CANCELLED);
        s->upq.clear();
    }
    free_server(s);
    delete s;
}

}  // extern "C"
