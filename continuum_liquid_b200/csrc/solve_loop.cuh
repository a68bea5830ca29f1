// The tolerance-mode iteration as one CUDA graph that loops on the device (no counterpart in the
// reference, whose pressure solve runs a fixed number of W-cycles, pressure_solve.py:61-84).
//
// A host loop has to read the residual to decide whether to run another refinement; each read drains
// the device and leaves it idle while the host decides and launches the next batch. Here the decision
// is a node of the graph: a WHILE conditional node whose body is
//     refinement (FP64 buffers 0 -> 1), check, IF { refinement (1 -> 0), check }
// where a refinement is the W-cycle on the residual followed by the FCG dots and step (or the plain
// refinement step), and the check -- one thread -- counts the refinement, records its relative
// residual and sets both conditions to (residual > tol and refinements < max). The IF makes the loop
// stop after the refinement that reaches the tolerance, whichever of the pair it is, and the two
// halves alternate the buffers as the host loop does. The count is capped, so the loop always ends.
// Included by clb200.cu inside its extern "C" block (helpers are C++).
extern "C++" {
namespace clb {

// One thread: the refinement just run is number ++*cycles; history[cycles] = its relative residual
// sqrt(sum r^2 / sum b^2) (as the host computes it); both conditions = whether to go on.
__global__ void k_loop_check(const double* __restrict__ norms, double tol, int max_cycles, int* __restrict__ cycles,
                             double* __restrict__ history, int history_len, cudaGraphConditionalHandle h_while,
                             cudaGraphConditionalHandle h_if, int set_if) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int c = *cycles + 1;
    *cycles = c;
    const double rr = norms[0], bb = norms[1];
    const double rel = bb == 0.0 ? 0.0 : sqrt(rr / bb);
    if (c < history_len) history[c] = rel;
    const unsigned go = (rel > tol && c < max_cycles) ? 1u : 0u;
    cudaGraphSetConditional(h_while, go);
    if (set_if) cudaGraphSetConditional(h_if, go);
}

// Before the loop: the WHILE node's condition defaults to 0 and this kernel sets it to 1, so a
// condition that could not be set leaves the loop body unrun rather than running without end.
__global__ void k_loop_start(cudaGraphConditionalHandle h_while) {
    if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(h_while, 1u);
}

}  // namespace clb
}  // extern "C++"

struct clb_solve_loop {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int launches_per_refinement;
};

extern "C++" {
namespace {

struct LoopBuffers {
    float *correction, *residual, *direction[2];
    double *p64[2], *fcg_state, *norms;
    const float* rhs;
    void *fcg_partials, *partials;
    int method, pre, post, coarse;
};

int loop_refinement(const clb_mg_hierarchy* h, const LoopBuffers& a, int src, cudaStream_t s) {
    const int* n = h->shape[0];
    if (clb_mg_w_cycle(h, a.correction, a.residual, a.pre, a.post, a.coarse, s)) return 1;
    if (a.method == 0) {
        if (clb_mg_fcg_dots(a.correction, a.direction[src], a.residual, h->op0, h->delta, n[0], n[1], n[2],
                            a.fcg_partials, a.fcg_state, s))
            return 1;
        return clb_mg_fcg_step(a.p64[src], a.correction, a.direction[src], a.p64[1 - src], a.direction[1 - src],
                               a.fcg_state, a.rhs, h->op0, h->delta, n[0], n[1], n[2], a.residual, a.partials,
                               a.norms, s);
    }
    return clb_mg_ir_step(a.p64[src], a.correction, a.p64[1 - src], a.rhs, h->op0, h->delta, n[0], n[1], n[2],
                          a.residual, a.partials, a.norms, s);
}

// Captures refinement `src` and its check into `body` (a conditional node's body graph) on stream s;
// *check_out: the check's node (the last node of the body).
int capture_half(const clb_mg_hierarchy* h, const LoopBuffers& a, int src, cudaGraph_t body, cudaStream_t s,
                 double tol, int max_cycles, int* cycles, double* history, int history_len,
                 cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hi, int set_if, cudaGraphNode_t* check_out) {
    if (check_call(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                   "solve loop: begin capture"))
        return 1;
    int err = loop_refinement(h, a, src, s);
    if (!err) {
        k_loop_check<<<1, 32, 0, s>>>(a.norms, tol, max_cycles, cycles, history, history_len, hw, hi, set_if);
        err = check_launch("k_loop_check");
    }
    if (!err && check_out) {
        cudaStreamCaptureStatus status;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        err = check_call(cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &ndeps), "solve loop: capture info");
        if (!err && ndeps != 1) err = set_error("solve loop: %zu capture dependencies after the check", ndeps);
        if (!err) *check_out = deps[0];
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s, &captured);
    if (err) return 1;
    return check_call(end, "solve loop: end capture");
}

}  // namespace
}  // extern "C++"

extern "C++" {
namespace {
int build_loop(const clb_mg_hierarchy& hz, const LoopBuffers& a, double tol, int max_cycles, int* cycles,
               double* history, int history_len, clb_solve_loop** out) {
    cudaStream_t s = nullptr;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    int err = check_call(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "solve loop: stream");
    if (!err) err = check_call(cudaGraphCreate(&g, 0), "solve loop: graph");
    cudaGraphConditionalHandle hw{}, hi{};
    cudaGraph_t body_w = nullptr, body_i = nullptr;
    if (!err) err = check_call(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault), "solve loop: handle");
    // the start kernel, then the WHILE node after it
    cudaGraphNode_t start = nullptr;
    if (!err) {
        err = check_call(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                         "solve loop: begin capture");
        if (!err) {
            k_loop_start<<<1, 32, 0, s>>>(hw);
            err = check_launch("k_loop_start");
            cudaStreamCaptureStatus status;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            if (!err)
                err = check_call(cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &ndeps),
                                 "solve loop: capture info");
            if (!err && ndeps != 1) err = set_error("solve loop: %zu capture dependencies after the start", ndeps);
            if (!err) start = deps[0];
            cudaGraph_t captured = nullptr;
            const cudaError_t end = cudaStreamEndCapture(s, &captured);
            if (!err) err = check_call(end, "solve loop: end capture");
        }
    }
    if (!err) {
        cudaGraphNodeParams wp = {};
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        err = check_call(cudaGraphAddNode(&wnode, g, &start, 1, &wp), "solve loop: while node");
        if (!err) body_w = wp.conditional.phGraph_out[0];
    }
    if (!err)
        err = check_call(cudaGraphConditionalHandleCreate(&hi, body_w, 0, cudaGraphCondAssignDefault),
                         "solve loop: handle");
    const int64_t before = clb_launch_count();
    cudaGraphNode_t check0 = nullptr;
    if (!err)
        err = capture_half(&hz, a, 0, body_w, s, tol, max_cycles, cycles, history, history_len, hw, hi, 1, &check0);
    const int64_t per = clb_launch_count() - before;
    if (!err) {
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hi;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode;
        err = check_call(cudaGraphAddNode(&inode, body_w, &check0, 1, &ip), "solve loop: if node");
        if (!err) body_i = ip.conditional.phGraph_out[0];
    }
    if (!err) err = capture_half(&hz, a, 1, body_i, s, tol, max_cycles, cycles, history, history_len, hw, hi, 0, nullptr);
    if (!err) err = check_call(cudaGraphInstantiate(&exec, g, 0), "solve loop: instantiate");
    if (s) (void)cudaStreamDestroy(s);
    if (err) {
        if (g) (void)cudaGraphDestroy(g);
        (void)cudaGetLastError();
        return 1;
    }
    *out = new clb_solve_loop{g, exec, (int)per};
    return 0;
}
}  // namespace
}  // extern "C++"

int clb_solve_loop_create(const clb_mg_hierarchy* h, float* correction, float* residual, float* direction0,
                          float* direction1, double* p64_0, double* p64_1, const float* rhs, double* fcg_state,
                          void* fcg_partials, void* partials, double* norms, int method, int pre_smooth,
                          int post_smooth, int coarse_iterations, double tol, int max_cycles, int* cycles,
                          double* history, int history_len, clb_solve_loop** out) {
    if (check_hierarchy(h)) return 1;
    CLB_REQUIRE(out != nullptr, "solve_loop_create: null output");
    *out = nullptr;
    CLB_REQUIRE(correction && residual && p64_0 && p64_1 && rhs && partials && norms && cycles && history,
                "solve_loop_create: null pointer");
    CLB_REQUIRE(method == 0 || method == 1, "solve_loop_create: method %d is not 0 (FCG) or 1 (refinement)", method);
    CLB_REQUIRE(method == 1 || (direction0 && direction1 && fcg_state && fcg_partials),
                "solve_loop_create: FCG needs the directions, state and partials");
    CLB_REQUIRE(max_cycles >= 1 && max_cycles <= 100000, "solve_loop_create: max_cycles %d outside 1..100000",
                max_cycles);
    CLB_REQUIRE(pre_smooth >= 0 && post_smooth >= 0 && coarse_iterations >= 0, "solve_loop_create: negative sweeps");
    CLB_REQUIRE(tol > 0.0, "solve_loop_create: tolerance must be positive");
    // the W-cycles of the loop start from a zero correction that the buffer does not hold (as the host loop)
    clb_mg_hierarchy hz = *h;
    hz.zero_outside = 2;
    const LoopBuffers a{correction, residual, {direction0, direction1}, {p64_0, p64_1}, fcg_state, norms, rhs,
                        fcg_partials, partials, method, pre_smooth, post_smooth, coarse_iterations};
    if (build_loop(hz, a, tol, max_cycles, cycles, history, history_len, out) == 0) return 0;
    if (!g_use_pdl) return 1;
    // a driver that takes no programmatic edges inside conditional bodies: the same graph without them
    g_use_pdl = false;
    const int err = build_loop(hz, a, tol, max_cycles, cycles, history, history_len, out);
    g_use_pdl = true;
    return err;
}

int clb_solve_loop_launch(clb_solve_loop* loop, int* cycles, void* stream) {
    CLB_REQUIRE(loop != nullptr && cycles != nullptr, "solve_loop_launch: null argument");
    cudaStream_t s = CLB_STREAM(stream);
    if (check_call(cudaMemsetAsync(cycles, 0, sizeof(int), s), "solve loop: reset count")) return 1;
    return check_call(cudaGraphLaunch(loop->exec, s), "solve loop: launch");
}

int clb_solve_loop_launches(const clb_solve_loop* loop) { return loop ? loop->launches_per_refinement : 0; }

int clb_solve_loop_destroy(clb_solve_loop* loop) {
    if (!loop) return 0;
    int err = 0;
    if (loop->exec) err |= check_call(cudaGraphExecDestroy(loop->exec), "solve loop: destroy exec");
    if (loop->graph) err |= check_call(cudaGraphDestroy(loop->graph), "solve loop: destroy graph");
    delete loop;
    return err;
}
