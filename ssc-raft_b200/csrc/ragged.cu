// ragged.cu -- a batch of independent reconstruction requests of different
// sizes and angle counts (FBP and emission EM), run together on one GPU.
//
// The reference reconstructs one call at a time and one size per call
// (getFBPMultiGPU / get_eEM_RT_MultiGPU); a server with mixed requests would
// loop over them.  Here:
//   * FBP requests: one filter launch per request, then ONE persistent
//     backprojector launch over every (request, tile) work item, queued
//     shortest request first;
//   * eEM requests: the sensitivity images in one persistent launch, then the
//     whole iteration loop -- one ragged projector launch and one persistent
//     backprojector-with-update launch per iteration over all EM requests --
//     captured once as a CUDA graph and replayed;
//   * the FBP and EM halves run concurrently on two streams, FBP at high
//     priority so short FBP requests are not queued behind EM iterations;
//   * each request's completion time is stamped on the device (%globaltimer)
//     by the CTA that finishes its last work item, giving per-request latency.
#include "engine.hpp"

#include <algorithm>
#include <numeric>
#include <vector>

#include "../../include/raft_b200.h"

namespace raft {

namespace {

// Byte offsets into the batch workspace (every region is assigned by the
// layout loop below; they start at zero only so that none is ever undefined).
struct FbpReq {
    int idx = 0;
    FbpPrepared fp;
    size_t tab = 0, rows = 0;
    double cost = 0.0;
};

struct EmReq {
    int idx = 0;
    EmPrepared ep;
    size_t tab = 0, rows = 0, den = 0, imgT = 0;
    double cost = 0.0;
};

size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace raft

using namespace raft;

extern "C" int raft_ragged_device(int gpu, const raft_request *reqs, int nreq, int geometry, int store,
                                  double *latency_ms, double *total_ms, void *stream)
{
    clear_error();
    if (!reqs || nreq < 1) {
        set_error("raft_ragged_device: empty request list");
        return 1;
    }
    if (!check_gpu_id(gpu)) return 1;
    if ((geometry == GEOM_FBP_REF && store != STORE_F32) ||
        (geometry == GEOM_FBP_LIN && store != STORE_PAIR_F32 && store != STORE_PAIR_BF16) ||
        (geometry != GEOM_FBP_REF && geometry != GEOM_FBP_LIN)) {
        set_error("raft_ragged_device: geometry/store as raft_fbp_ext (0/0, 1/1, 1/2)");
        return 1;
    }
    int em_iters = -1;
    for (int i = 0; i < nreq; i++) {
        const raft_request &q = reqs[i];
        if ((q.kind != 0 && q.kind != 1) || q.nrays < 2 || q.nrays > 65536 || q.nangles < 2 || !q.angles ||
            !q.d_data || !q.d_out) {
            set_error("raft_ragged_device: request " + std::to_string(i) + " is invalid");
            return 1;
        }
        if (q.kind == 0 && (q.pad < 0 || q.pad > 64 || q.filter < 0 || q.filter > 9 || !(q.pixel > 0.f))) {
            set_error("raft_ragged_device: FBP request " + std::to_string(i) + " has invalid parameters");
            return 1;
        }
        if (q.kind == 1) {
            if (q.niter < 0 || (em_iters >= 0 && q.niter != em_iters)) {
                set_error("raft_ragged_device: all eEM requests of a batch need the same iteration count");
                return 1;
            }
            em_iters = q.niter;
        }
    }
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        // s0: caller's stream (or the high-priority one) for FBP; s1: low-priority EM
        cudaStream_t s0 = resolve_stream(ds, stream, ds.s_hi);
        cudaStream_t s1 = ds.s_lo;

        // ---- plan every request and lay out one workspace ----------------
        std::vector<FbpReq> F;
        std::vector<EmReq> E;
        size_t off = a256(sizeof(unsigned long long) + sizeof(int));   // stamp + error flag
        for (int i = 0; i < nreq; i++) {
            const raft_request &q = reqs[i];
            const int N = q.nrays, A = q.nangles;
            if (q.kind == 0) {
                FbpConfig c;
                c.nrays = N;
                c.nangles = A;
                c.nslices = 1;
                c.objsize = N;
                c.pad = q.pad;
                c.filter = q.filter;
                c.pixel_x = c.pixel_y = q.pixel;
                c.offset = q.offset;
                c.geometry = geometry;
                c.store = store;
                FbpReq r;
                r.idx = i;
                r.fp = prepare_fbp(c, gpu);
                r.tab = off;
                off = a256(off + sizeof(double) * 2 * A + sizeof(float) * 4 * A);
                r.rows = off;
                off = a256(off + fbp_rows_bytes(r.fp, 1));
                r.cost = (double)N * N * A;
                F.push_back(r);
            } else {
                EmConfig c;
                c.nrays = N;
                c.nangles = A;
                c.nslices = 1;
                c.objsize = N;
                c.niter = q.niter;
                EmReq r;
                r.idx = i;
                r.ep = prepare_em(c);
                r.tab = off;
                off = a256(off + sizeof(float) * 4 * A);
                r.rows = off;
                off = a256(off + sizeof(float) * (size_t)A * r.ep.win.Wg);
                r.den = off;
                off = a256(off + sizeof(float) * (size_t)N * N);
                r.imgT = off;                      // transposed iterate for the projector's steep angles
                off = a256(off + sizeof(float) * (size_t)N * N);
                r.cost = 2.0 * N * N * A * q.niter;
                E.push_back(r);
            }
        }
        // shortest request first in the work queues (lower median latency)
        std::sort(F.begin(), F.end(), [](const FbpReq &a, const FbpReq &b) { return a.cost < b.cost; });
        std::sort(E.begin(), E.end(), [](const EmReq &a, const EmReq &b) { return a.cost < b.cost; });
        const size_t o_rb_fbp = off;
        off = a256(off + ragged_bp_bytes((int)F.size()));
        const size_t o_rb_den = off;
        off = a256(off + ragged_bp_bytes((int)E.size()));
        const size_t o_rb_upd = off;
        off = a256(off + ragged_bp_bytes((int)E.size()));
        const size_t o_proj = off;
        off = a256(off + sizeof(ProjLaunch) * E.size());
        const size_t o_blk = off;
        off = a256(off + sizeof(int) * (E.size() + 1));
        char *ws = (char *)ds.rows.get(off);
        unsigned long long *d_t0 = (unsigned long long *)ws;
        int *d_err = (int *)(ws + sizeof(unsigned long long));
        RAFT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s0));

        // ---- tables (not part of the timed region) ----------------------
        std::vector<BpLaunch> bF(F.size()), bD(E.size()), bU(E.size());
        std::vector<const float *> wtF(F.size());
        std::vector<ProjLaunch> P(E.size());
        std::vector<int> blk(E.size() + 1, 0);
        for (size_t k = 0; k < F.size(); k++) {
            const raft_request &q = reqs[F[k].idx];
            const int A = q.nangles;
            char *t = ws + F[k].tab;
            FbpTables tb;
            tb.csd = (double *)t;
            tb.snd = tb.csd + A;
            float *d_ang = (float *)(tb.snd + A);
            tb.cs = d_ang + A;
            tb.sn = tb.cs + A;
            tb.wt = tb.sn + A;
            tb.err = d_err;
            wtF[k] = tb.wt;
            RAFT_CUDA(cudaMemcpy(d_ang, q.angles, sizeof(float) * A, cudaMemcpyHostToDevice));
            launch_angle_tables(d_ang, A, tb.cs, tb.sn, tb.wt, 0, s0);
            if (geometry == GEOM_FBP_LIN) {
                std::vector<double> cd(2 * (size_t)A);
                for (int a = 0; a < A; a++) {
                    cd[a] = std::cos((double)q.angles[a]);
                    cd[A + a] = std::sin((double)q.angles[a]);
                }
                RAFT_CUDA(cudaMemcpy(tb.csd, cd.data(), sizeof(double) * 2 * A, cudaMemcpyHostToDevice));
            }
            BpLaunch &b = bF[k];
            b.filt = ws + F[k].rows;
            b.img = q.d_out;
            b.No = q.nrays;
            b.nangles = A;
            b.nslices = 1;
            b.geometry = geometry;
            b.store = store;
            b.win = F[k].fp.win;
            b.geo = F[k].fp.geo;
            b.cs = tb.cs;
            b.sn = tb.sn;
            b.csd = tb.csd;
            b.snd = tb.snd;
            b.err = d_err;
        }
        for (size_t k = 0; k < E.size(); k++) {
            const raft_request &q = reqs[E[k].idx];
            const int A = q.nangles, N = q.nrays;
            float *d_ang = (float *)(ws + E[k].tab);
            float *cs = d_ang + A, *sn = cs + A, *wt = sn + A;
            RAFT_CUDA(cudaMemcpy(d_ang, q.angles, sizeof(float) * A, cudaMemcpyHostToDevice));
            launch_angle_tables(d_ang, A, cs, sn, wt, 1, s0);
            float *rows = (float *)(ws + E[k].rows);
            RAFT_CUDA(cudaMemsetAsync(rows, 0, sizeof(float) * (size_t)A * E[k].ep.win.Wg, s0));
            BpLaunch b;
            b.filt = rows;
            b.No = N;
            b.nangles = A;
            b.nslices = 1;
            b.geometry = GEOM_EM_REF;
            b.store = STORE_F32;
            b.win = E[k].ep.win;
            b.geo = E[k].ep.geo;
            b.cs = cs;
            b.sn = sn;
            b.err = d_err;
            bD[k] = b;
            bD[k].img = (float *)(ws + E[k].den);
            bU[k] = b;
            bU[k].img = q.d_out;
            bU[k].den = (const float *)(ws + E[k].den);
            ProjLaunch &p = P[k];
            p.img = q.d_out;
            p.imgT = (const float *)(ws + E[k].imgT);   // transposed copy for steep angles
            p.out = rows;
            p.angles = d_ang;
            p.nx = p.ny = p.nrays = N;
            p.nangles = A;
            p.nslices = 1;
            p.em = 1;
            p.epilogue = 2;
            p.data = q.d_data;
            p.wt = wt;
            p.windowed = 1;
            p.wlo = E[k].ep.win.wlo;
            p.Wg = E[k].ep.win.Wg;
            blk[k + 1] = blk[k] + project_blocks_per_slice(N, A);
        }
        RaggedBp rbF, rbD, rbU;
        if (!F.empty()) ragged_bp_prepare(rbF, bF.data(), (int)F.size(), geometry, store, ws + o_rb_fbp);
        if (!E.empty()) {
            ragged_bp_prepare(rbD, bD.data(), (int)E.size(), GEOM_EM_REF, STORE_F32, ws + o_rb_den);
            ragged_bp_prepare(rbU, bU.data(), (int)E.size(), GEOM_EM_REF, STORE_F32, ws + o_rb_upd);
            RAFT_CUDA(cudaMemcpy(ws + o_proj, P.data(), sizeof(ProjLaunch) * E.size(), cudaMemcpyHostToDevice));
            RAFT_CUDA(cudaMemcpy(ws + o_blk, blk.data(), sizeof(int) * (E.size() + 1), cudaMemcpyHostToDevice));
        }
        // the EM iteration loop as one graph (captured before the timed region)
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        if (!E.empty() && em_iters > 0) {
            RAFT_CUDA(cudaStreamBeginCapture(s1, cudaStreamCaptureModeThreadLocal));
            try {
                for (int it = 0; it < em_iters; it++) {
                    for (size_t k = 0; k < E.size(); k++)
                        launch_transpose(reqs[E[k].idx].d_out, (float *)P[k].imgT, P[k].nx, P[k].nx, 1, s1);
                    launch_project_ragged((const ProjLaunch *)(ws + o_proj), (const int *)(ws + o_blk),
                                          (int)E.size(), blk.back(), 1, 2, s1);
                    ragged_bp_launch(rbU, s1);
                }
            } catch (...) {
                cudaStreamEndCapture(s1, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            RAFT_CUDA(cudaStreamEndCapture(s1, &graph));
            RAFT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        }
        RAFT_CUDA(cudaStreamSynchronize(s0));

        // ---- timed region: everything from here runs on the device -------
        cudaEvent_t e0, e1;
        RAFT_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
        RAFT_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
        launch_stamp(d_t0, s0);
        RAFT_CUDA(cudaEventRecord(e0, s0));
        RAFT_CUDA(cudaStreamWaitEvent(s1, e0, 0));
        for (size_t k = 0; k < F.size(); k++) {
            const raft_request &q = reqs[F[k].idx];
            FilterLaunch fl;
            fl.sino = q.d_data;
            fl.out = const_cast<void *>(bF[k].filt);
            fl.wt = wtF[k];
            fl.nrows = q.nangles;
            fl.nangles = q.nangles;
            fl.wlo = F[k].fp.win.wlo;
            fl.Wg = F[k].fp.win.Wg;
            fl.store = geometry == GEOM_FBP_LIN ? store : STORE_F32;
            launch_filter(*F[k].fp.plan, fl, s0);
        }
        if (!F.empty()) ragged_bp_launch(rbF, s0);
        if (!E.empty()) {
            for (size_t k = 0; k < E.size(); k++) {
                const raft_request &q = reqs[E[k].idx];
                launch_to_window(nullptr, (float *)bD[k].filt, P[k].wt, q.nangles, q.nangles, q.nrays,
                                 E[k].ep.win.wlo, E[k].ep.win.Wg, s1);
            }
            ragged_bp_launch(rbD, s1);
            if (exec) RAFT_CUDA(cudaGraphLaunch(exec, s1));
        }
        RAFT_CUDA(cudaEventRecord(e1, s1));
        RAFT_CUDA(cudaStreamWaitEvent(s0, e1, 0));
        RAFT_CUDA(cudaStreamSynchronize(s0));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);

        // ---- latencies -----------------------------------------------------
        unsigned long long t0 = 0;
        int flag = 0;
        RAFT_CUDA(cudaMemcpy(&t0, d_t0, sizeof(t0), cudaMemcpyDeviceToHost));
        RAFT_CUDA(cudaMemcpy(&flag, d_err, sizeof(int), cudaMemcpyDeviceToHost));
        RAFT_CHECK(flag == 0, "raft_ragged_device: a bounded wait in the staging pipeline timed out");
        std::vector<unsigned long long> tf(F.size()), te(E.size());
        if (!F.empty())
            RAFT_CUDA(cudaMemcpy(tf.data(), rbF.d_tdone, sizeof(unsigned long long) * F.size(), cudaMemcpyDeviceToHost));
        if (!E.empty()) {
            const unsigned long long *src = em_iters > 0 ? rbU.d_tdone : rbD.d_tdone;
            RAFT_CUDA(cudaMemcpy(te.data(), src, sizeof(unsigned long long) * E.size(), cudaMemcpyDeviceToHost));
        }
        double tmax = 0.0;
        for (size_t k = 0; k < F.size(); k++) {
            const double ms = tf[k] > t0 ? (tf[k] - t0) * 1e-6 : 0.0;
            if (latency_ms) latency_ms[F[k].idx] = ms;
            tmax = std::max(tmax, ms);
        }
        for (size_t k = 0; k < E.size(); k++) {
            const double ms = te[k] > t0 ? (te[k] - t0) * 1e-6 : 0.0;
            if (latency_ms) latency_ms[E[k].idx] = ms;
            tmax = std::max(tmax, ms);
        }
        if (total_ms) *total_ms = tmax;
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}
