// qk_dist.cpp -- NCCL communicators and the sharded execution of a plan
// (see qk_dist.h).  No counterpart in the reference, which prices on one host.
#include "qk_dist.h"

#include <dlfcn.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <nccl.h>

#include "../../include/qk_api.h"
#include "mc_plan.h"
#include "qk_error.h"
#include "qk_fault.h"

namespace {

// The NCCL entry points the library uses, resolved once per process.
struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*comm_abort)(ncclComm_t) = nullptr;
    ncclResult_t (*broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t,
                               ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
    std::string load_error;
};

const NcclApi& nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* path = std::getenv("QK_B200_NCCL_PATH");
        void* h = dlopen(path && *path ? path : "libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            const char* e = dlerror();
            api.load_error = e ? e : "dlopen failed";
            return;
        }
        auto sym = [&](const char* name) {
            void* f = dlsym(h, name);
            if (!f && api.load_error.empty()) api.load_error = std::string("missing ") + name;
            return f;
        };
        api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
        api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(sym("ncclCommInitRank"));
        api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
        api.comm_abort = reinterpret_cast<decltype(api.comm_abort)>(sym("ncclCommAbort"));
        api.broadcast = reinterpret_cast<decltype(api.broadcast)>(sym("ncclBroadcast"));
        api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(sym("ncclAllReduce"));
        api.group_start = reinterpret_cast<decltype(api.group_start)>(sym("ncclGroupStart"));
        api.group_end = reinterpret_cast<decltype(api.group_end)>(sym("ncclGroupEnd"));
        api.error_string = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
    });
    return api;
}

int32_t nccl_missing(const char* where) {
    qkb::set_error_fmt("nccl unavailable: %s in %s", nccl().load_error.c_str(), where);
    return QK_ERR_RUNTIME_INIT;
}

int32_t fail_nccl(ncclResult_t r, const char* where) {
    qkb::set_error_fmt("nccl error: %s in %s", nccl().error_string ? nccl().error_string(r) : "?",
                       where);
    return QK_ERR_RUNTIME_INIT;
}

}  // namespace

struct qk_dist {
    ncclComm_t comm = nullptr;
    int world = 0;
    int rank = 0;
    int device = -1;
    int64_t* d_check = nullptr;  // 4 int64 on `device`: the tiling check
    // set by qk_dist_abort (possibly from another thread); NCCL frees an
    // aborted communicator, so no call may use `comm` afterwards
    std::atomic<bool> aborted{false};
};

namespace {

// A fingerprint of the plan's tiling and partition (62 bits, so its negation
// stays in range): every rank must hold the same one before tile sums move.
int64_t tiling_fingerprint(qkb::Plan& plan, const std::vector<int64_t>& b) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the words below
    auto mix = [&h](uint64_t v) {
        for (int i = 0; i < 8; ++i) {
            h ^= (v >> (8 * i)) & 0xFF;
            h *= 1099511628211ull;
        }
    };
    mix((uint64_t)plan.n());
    mix((uint64_t)plan.n_tiles());
    mix((uint64_t)plan.block());
    mix((uint64_t)(int64_t)plan.upt());
    for (int64_t x : b) mix((uint64_t)x);
    return (int64_t)(h >> 2);
}

}  // namespace

namespace qkb {

int32_t dist_execute(Plan& plan, qk_dist* d, cudaStream_t stream, const char* where) {
    if (!d) return fail_null("dist");
    if (!nccl().load_error.empty()) return nccl_missing(where);
    if (d->aborted.load()) {
        set_error_fmt("invalid input: the communicator was aborted in %s", where);
        return QK_ERR_INVALID_INPUT;
    }
    if (plan.device() != d->device) {
        set_error_fmt("invalid input: plan on device %d, communicator on device %d in %s",
                      plan.device(), d->device, where);
        return QK_ERR_INVALID_INPUT;
    }
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != d->device) e = cudaSetDevice(d->device);
    if (e != cudaSuccess) return fail_cuda(e, where);
    cudaStream_t st = stream ? stream : plan.stream();
    int32_t rc = QK_OK;
    const std::vector<int64_t>& b = plan.shard_bounds(d->world);
    e = plan.order_after_upload(st);
    // Every rank must hold the same tiling, or the broadcasts below would
    // disagree in size: max-reduce (n_tiles, fingerprint, -n_tiles,
    // -fingerprint); all ranks see the same result and fail alike.
    if (e == cudaSuccess) {
        const int64_t fp = tiling_fingerprint(plan, b);
        int64_t v[4] = {plan.n_tiles(), fp, -plan.n_tiles(), -fp};
        e = cudaMemcpyAsync(d->d_check, v, sizeof v, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            const ncclResult_t r = nccl().all_reduce(d->d_check, d->d_check, 4, ncclInt64, ncclMax,
                                                     d->comm, st);
            if (r != ncclSuccess) {
                if (prev >= 0 && prev != d->device) cudaSetDevice(prev);
                return fail_nccl(r, where);
            }
            e = cudaMemcpyAsync(v, d->d_check, sizeof v, cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && (v[0] != -v[2] || v[1] != -v[3])) {
            if (prev >= 0 && prev != d->device) cudaSetDevice(prev);
            set_error_fmt("invalid input: the ranks hold different tilings of the batch (same "
                          "inputs, flags and launch shape on every rank) in %s", where);
            return QK_ERR_INVALID_INPUT;
        }
    }
    if (e != cudaSuccess) {
        if (prev >= 0 && prev != d->device) cudaSetDevice(prev);
        return fail_cuda(e, where);
    }
    // A failed launch on this rank still takes part in the exchange below, so
    // that no other rank waits for it; it reports its error afterwards.
    const cudaError_t e_sim = plan.launch_tiles(st, b[(size_t)d->rank], b[(size_t)d->rank + 1], false);
    if ((e = injected_fault(kFaultCollective)) != cudaSuccess) {
        rc = fail_cuda(e, where);
    } else {
        // every rank's tile range of partials to every rank: one broadcast per
        // rank (in place at the root), one grouped collective step; all ranks
        // compute the same bounds, so they issue the same calls in the same order
        TilePartial* parts = plan.d_partials();
        ncclResult_t r = nccl().group_start();
        for (int k = 0; k < d->world && r == ncclSuccess; ++k) {
            const int64_t lo = b[(size_t)k], hi = b[(size_t)k + 1];
            if (hi <= lo) continue;
            r = nccl().broadcast(parts + lo, parts + lo, (size_t)(hi - lo) * sizeof(TilePartial),
                                 ncclUint8, k, d->comm, st);
        }
        const ncclResult_t r_end = nccl().group_end();
        if (r == ncclSuccess) r = r_end;
        if (r != ncclSuccess) rc = fail_nccl(r, where);
    }
    if (rc == QK_OK && e_sim != cudaSuccess) rc = fail_cuda(e_sim, where);
    if (rc == QK_OK) {
        e = plan.launch_finalize_all(st);
        if (e != cudaSuccess) rc = fail_cuda(e, where);
    }
    if (rc == QK_OK) plan.note_stream(st);
    if (prev >= 0 && prev != d->device) cudaSetDevice(prev);
    return rc;
}

}  // namespace qkb

extern "C" {

int32_t qk_dist_unique_id(uint8_t* out_id) {
    if (!out_id) return qkb::fail_null("out_id");
    if (!nccl().load_error.empty()) return nccl_missing("qk_dist_unique_id");
    static_assert(sizeof(ncclUniqueId) == QK_DIST_ID_BYTES, "NCCL unique id size");
    ncclUniqueId id;
    const ncclResult_t r = nccl().get_unique_id(&id);
    if (r != ncclSuccess) return fail_nccl(r, "qk_dist_unique_id");
    std::memcpy(out_id, &id, sizeof id);
    return QK_OK;
}

int32_t qk_dist_create(const uint8_t* id, int32_t world, int32_t rank, qk_dist** out) {
    if (!id) return qkb::fail_null("id");
    if (!out) return qkb::fail_null("out");
    *out = nullptr;
    if (world <= 0) return qkb::fail_size(world);
    if (rank < 0 || rank >= world) {
        qkb::set_error_fmt("invalid input: rank %d of world %d", rank, world);
        return QK_ERR_INVALID_INPUT;
    }
    if (!nccl().load_error.empty()) return nccl_missing("qk_dist_create");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return qkb::fail_cuda(e, "qk_dist_create");
    ncclUniqueId uid;
    std::memcpy(&uid, id, sizeof uid);
    qk_dist* d = new qk_dist();
    e = cudaMalloc(&d->d_check, 4 * sizeof(int64_t));
    if (e != cudaSuccess) {
        delete d;
        return qkb::fail_cuda(e, "qk_dist_create");
    }
    const ncclResult_t r = nccl().comm_init_rank(&d->comm, world, uid, rank);
    if (r != ncclSuccess) {
        cudaFree(d->d_check);
        delete d;
        return fail_nccl(r, "qk_dist_create");
    }
    d->world = world;
    d->rank = rank;
    d->device = dev;
    *out = d;
    return QK_OK;
}

int32_t qk_dist_info(const qk_dist* d, int32_t* world, int32_t* rank, int32_t* device) {
    if (!d) return qkb::fail_null("dist");
    if (world) *world = d->world;
    if (rank) *rank = d->rank;
    if (device) *device = d->device;
    return QK_OK;
}

int32_t qk_dist_abort(qk_dist* d) {
    if (!d) return qkb::fail_null("dist");
    if (d->aborted.exchange(true)) return QK_OK;  // already aborted
    const ncclResult_t r = nccl().comm_abort(d->comm);
    return r == ncclSuccess ? QK_OK : fail_nccl(r, "qk_dist_abort");
}

int32_t qk_dist_destroy(qk_dist* d) {
    if (!d) return QK_OK;
    ncclResult_t r = ncclSuccess;
    if (d->comm && !d->aborted.load()) r = nccl().comm_destroy(d->comm);
    if (d->d_check) {
        int prev = -1;
        if (cudaGetDevice(&prev) == cudaSuccess && prev != d->device) cudaSetDevice(d->device);
        cudaFree(d->d_check);
        if (prev >= 0 && prev != d->device) cudaSetDevice(prev);
    }
    delete d;
    return r == ncclSuccess ? QK_OK : fail_nccl(r, "qk_dist_destroy");
}

int32_t qk_dist_partition(const double* cost, int64_t n, int32_t world, int64_t* bounds) {
    if (!cost && n > 0) return qkb::fail_null("cost");
    if (!bounds) return qkb::fail_null("bounds");
    if (world <= 0 || n < 0) return qkb::fail_size(world <= 0 ? world : n);
    qkb::partition_by_cost(cost, n, world, bounds);
    return QK_OK;
}

}  // extern "C"
