// Per-step PLY export without stalling the GPU (the reference's drivers export every step with
// Simulation::export_mesh -> export_ply_float, MeshIO.cpp:263-298).  The file layout is that
// writer's: a text header, then per vertex float32 x, y, z, phi, psi, then per face a uchar 3 and
// three uint32 indices.
//
// bem_export_ply_async packs the device state into float32 records (one kernel on the context's
// stream, so the next step may overwrite the state right after it), copies them to pinned memory on
// a separate copy stream, and hands the file to a writer thread that waits for that copy.  A ring of
// slots bounds the memory; when all are in flight the call waits for the oldest.  bem_export_wait
// returns when every queued file is written (and reports the first write error).
#include <stdio.h>
#include <string.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"

namespace bemb {

struct PlyRec {
    float x, y, z, phi, psi;
};
static_assert(sizeof(PlyRec) == 20, "packed float32 vertex record");

__global__ void k_pack_ply(int N, const double* __restrict__ x, const double* __restrict__ phi,
                           const double* __restrict__ psi, PlyRec* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[i] = {__double2float_rn(x[3 * i]), __double2float_rn(x[3 * i + 1]), __double2float_rn(x[3 * i + 2]),
              __double2float_rn(phi[i]), __double2float_rn(psi[i])};
}

struct PlyExporter {
    static constexpr int SLOTS = 4;
    struct Slot {
        PlyRec* dev = nullptr;
        PlyRec* host = nullptr;
        cudaEvent_t packed = nullptr, copied = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        std::string path;
    };
    int device = 0;
    int64_t N = 0;
    std::vector<uint32_t> tri;  // M*3
    cudaStream_t copy = nullptr;
    Slot slots[SLOTS];
    int next = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> jobs;
    bool stop = false;
    int pending = 0;
    std::string error;
    std::thread worker;

    void run() {
        cudaSetDevice(device);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                j = jobs.front();
                jobs.pop_front();
            }
            Slot& s = slots[j.slot];
            std::string err;
            if (cudaEventSynchronize(s.copied) != cudaSuccess) err = "export: device copy failed";
            if (err.empty()) err = write(j.path, s.host);
            std::lock_guard<std::mutex> lk(mu);
            s.busy = false;
            --pending;
            if (!err.empty() && error.empty()) error = err;
            cv.notify_all();
        }
    }

    std::string write(const std::string& path, const PlyRec* v) const {
        FILE* f = fopen(path.c_str(), "wb");
        if (!f) return "export: cannot open " + path;
        const size_t m = tri.size() / 3;
        std::string head = "ply\nformat binary_little_endian 1.0\ncomment Output from BEM simulation\nelement vertex " +
                           std::to_string(N) +
                           "\nproperty float x\nproperty float y\nproperty float z\nproperty float phi\nproperty float "
                           "psi\nelement face " +
                           std::to_string(m) + "\nproperty list uchar uint vertex_indices\nend_header\n";
        bool ok = fwrite(head.data(), 1, head.size(), f) == head.size();
        ok = ok && fwrite(v, sizeof(PlyRec), (size_t)N, f) == (size_t)N;
        std::vector<unsigned char> faces(m * 13);
        for (size_t t = 0; t < m; ++t) {
            faces[13 * t] = 3;
            memcpy(&faces[13 * t + 1], &tri[3 * t], 12);
        }
        ok = ok && fwrite(faces.data(), 1, faces.size(), f) == faces.size();
        ok = (fclose(f) == 0) && ok;
        return ok ? std::string() : "export: write failed for " + path;
    }

    // wait for every queued file; returns (and clears) the first error
    std::string flush() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return pending == 0; });
        std::string e = error;
        error.clear();
        return e;
    }

    ~PlyExporter() {
        flush();
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        for (auto& s : slots) {
            cudaFree(s.dev);
            cudaFreeHost(s.host);
            if (s.packed) cudaEventDestroy(s.packed);
            if (s.copied) cudaEventDestroy(s.copied);
        }
        if (copy) cudaStreamDestroy(copy);
    }
};

void exporter_release(Ctx& c) {
    delete c.exporter;
    c.exporter = nullptr;
}

static int exporter_init(Ctx& c) {
    if (c.exporter && c.exporter->N == c.topo.N) return BEM_OK;
    exporter_release(c);
    auto* e = new (std::nothrow) PlyExporter();
    if (!e) return c.fail(BEM_ERR_NOMEM, "export: exporter");
    e->device = c.device;
    e->N = c.topo.N;
    e->tri.resize(c.h_tri.size());
    for (size_t k = 0; k < c.h_tri.size(); ++k) e->tri[k] = (uint32_t)c.h_tri[k];
    bool ok = cudaStreamCreateWithFlags(&e->copy, cudaStreamNonBlocking) == cudaSuccess;
    for (auto& s : e->slots) {
        ok = ok && cudaMalloc(&s.dev, sizeof(PlyRec) * (size_t)e->N) == cudaSuccess;
        ok = ok && cudaMallocHost(&s.host, sizeof(PlyRec) * (size_t)e->N) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&s.packed, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        delete e;
        return c.fail(BEM_ERR_NOMEM, "export: staging buffers");
    }
    e->worker = std::thread([e] { e->run(); });
    c.exporter = e;
    return BEM_OK;
}

int export_ply_async(Ctx& c, const char* path) {
    int rc = exporter_init(c);
    if (rc) return rc;
    PlyExporter& e = *c.exporter;
    const int k = e.next;
    {
        std::unique_lock<std::mutex> lk(e.mu);
        e.cv.wait(lk, [&] { return !e.slots[k].busy; });  // back-pressure: the oldest slot
        e.slots[k].busy = true;
        ++e.pending;
    }
    PlyExporter::Slot& s = e.slots[k];
    const int N = (int)c.topo.N;
    KLAUNCH(), k_pack_ply<<<(N + 255) / 256, 256, 0, c.stream>>>(N, c.x, c.phi, c.psi, s.dev);
    cudaError_t err = cudaEventRecord(s.packed, c.stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(e.copy, s.packed, 0);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(s.host, s.dev, sizeof(PlyRec) * (size_t)N, cudaMemcpyDeviceToHost, e.copy);
    if (err == cudaSuccess) err = cudaEventRecord(s.copied, e.copy);
    if (err != cudaSuccess) {
        std::lock_guard<std::mutex> lk(e.mu);
        s.busy = false;
        --e.pending;
        e.cv.notify_all();
        return c.fail(BEM_ERR_CUDA, std::string("export: ") + cudaGetErrorString(err));
    }
    e.next = (k + 1) % PlyExporter::SLOTS;
    {
        std::lock_guard<std::mutex> lk(e.mu);
        e.jobs.push_back({k, std::string(path)});
    }
    e.cv.notify_all();
    return BEM_OK;
}

int export_wait(Ctx& c) {
    if (!c.exporter) return BEM_OK;
    const std::string e = c.exporter->flush();
    if (!e.empty()) return c.fail(BEM_ERR_STATE, e);
    return BEM_OK;
}

}  // namespace bemb
