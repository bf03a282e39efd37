// Batched solves: many independent grids of uneven sizes and boundary
// conditions, replayed as one CUDA graph.
//
// The reference solves one grid per PencilDcmp object and launches every
// step separately (src/pencilDcmp.cpp:5801-6430).  Here each grid keeps a
// handle (plans, twiddles and workspaces resident on the device, zero-copy
// bound to the caller's RHS and solution buffers), the launch shape of each
// size class is chosen once by the autotuner, and the solves of all grids are
// captured into one graph whose branches run concurrently, so that small grids
// fill the GPU together and the whole batch costs one graph launch.
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pittpack_b200.h"

struct pp_batch_s {
    int device = 0;
    std::vector<pp_handle> handles;
    std::vector<cudaStream_t> branches;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int nodes = 0;  // graph nodes (kernels and memsets) per replay
};

namespace {

void batch_free(pp_batch_s* b)
{
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    // the handles name the branch streams: release them first
    for (auto h : b->handles) pp_destroy(h);
    for (auto s : b->branches) cudaStreamDestroy(s);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
}

// one handle per grid, tuned per size class, solved once outside the capture
int build_handles(pp_batch_s* b, const pp_batch_item* items, int n, const pp_options* opt, int autotune)
{
    // tuned launch shape per size class (nx, ny, nz, boundary letters)
    std::map<std::tuple<int, int, int, std::string>, pp_tuning> tuned;
    int rc = PP_SUCCESS;
    for (int i = 0; i < n && rc == PP_SUCCESS; ++i) {
        const pp_batch_item& it = items[i];
        pp_handle h = nullptr;
        if ((rc = pp_create(it.nx, it.ny, it.nz, &h)) != PP_SUCCESS) break;
        b->handles.push_back(h);
        if ((rc = pp_set_box(h, it.box)) != PP_SUCCESS) break;
        if ((rc = pp_assign_boundary(h, it.bc)) != PP_SUCCESS) break;
        if (opt && (rc = pp_set_options(h, opt)) != PP_SUCCESS) break;
        if (!it.d_rhs || !it.d_P) {
            rc = PP_INPUT_ARGS;
            break;
        }
        if ((rc = pp_bind_device_buffers(h, it.d_rhs, 0, it.d_P)) != PP_SUCCESS) break;
        const auto key = std::make_tuple(it.nx, it.ny, it.nz, std::string(it.bc, 6));
        const auto f = tuned.find(key);
        if (f != tuned.end()) {
            rc = pp_set_tuning(h, &f->second);
        } else if (autotune) {
            pp_tuning t;
            double ms = 0.0;
            if ((rc = pp_autotune(h, 3, &t, &ms)) == PP_SUCCESS) tuned[key] = t;
        }
        // one solve outside the capture: kernel attributes and lazily sized
        // buffers are set up before any launch is recorded
        if (rc == PP_SUCCESS) rc = pp_solve(h);
    }
    if (rc == PP_SUCCESS && cudaDeviceSynchronize() != cudaSuccess) rc = PP_CUDA_ERROR;
    return rc;
}

}  // namespace

extern "C" int pp_batch_create(const pp_batch_item* items, int n, const pp_options* opt, int branches, int autotune,
                               pp_batch* out)
{
    if (!items || n < 1 || !out || branches < 1 || branches > 64) return PP_INPUT_ARGS;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PP_GPU_INIT_FAILURE;
    pp_batch_s* b = new (std::nothrow) pp_batch_s;
    if (!b) return PP_ALLOCATION_FAIL;
    cudaGetDevice(&b->device);
    int rc = build_handles(b, items, n, opt, autotune);
    if (rc != PP_SUCCESS) {
        batch_free(b);
        return rc;
    }
    // capture: fork the grids over 'branches' streams, join, one graph
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    std::vector<cudaEvent_t> ev(branches + 1, nullptr);
    for (auto& x : ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    b->branches.assign(branches, nullptr);
    for (auto& s : b->branches)
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaEventRecord(ev[0], b->cap);
        for (auto s : b->branches) cudaStreamWaitEvent(s, ev[0], 0);
        for (int i = 0; i < n && rc == PP_SUCCESS; ++i) {
            if ((rc = pp_set_stream(b->handles[i], b->branches[i % branches])) == PP_SUCCESS)
                rc = pp_solve(b->handles[i]);
        }
        for (int k = 0; k < branches; ++k) {
            cudaEventRecord(ev[k + 1], b->branches[k]);
            cudaStreamWaitEvent(b->cap, ev[k + 1], 0);
        }
        // the capture is always ended, also after a failed solve
        const cudaError_t e2 = cudaStreamEndCapture(b->cap, &b->graph);
        if (e2 != cudaSuccess && rc == PP_SUCCESS) rc = PP_CUDA_ERROR;
    } else {
        rc = PP_CUDA_ERROR;
    }
    if (rc == PP_SUCCESS && cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) rc = PP_CUDA_ERROR;
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    if (rc != PP_SUCCESS) {
        batch_free(b);
        return rc;
    }
    size_t nodes = 0;
    cudaGraphGetNodes(b->graph, nullptr, &nodes);
    b->nodes = (int)nodes;
    *out = b;
    return PP_SUCCESS;
}

extern "C" int pp_batch_run(pp_batch b, void* stream)
{
    if (!b) return PP_INVALID_HANDLE;
    cudaSetDevice(b->device);
    return cudaGraphLaunch(b->exec, (cudaStream_t)stream) == cudaSuccess ? PP_SUCCESS : PP_CUDA_ERROR;
}

extern "C" int pp_batch_info(pp_batch b, int* grids, int* graph_nodes)
{
    if (!b) return PP_INVALID_HANDLE;
    if (grids) *grids = (int)b->handles.size();
    if (graph_nodes) *graph_nodes = b->nodes;
    return PP_SUCCESS;
}

extern "C" int pp_batch_destroy(pp_batch b)
{
    if (!b) return PP_INVALID_HANDLE;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    batch_free(b);
    return PP_SUCCESS;
}
