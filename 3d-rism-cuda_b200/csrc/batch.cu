// Batched solves of many small solutes (rism3d_solve_batch).  The reference
// solves one solute per process; here solutes with the same cubic cell are
// solved together in sub-batches of about batch_chunk_points grid points:
// every pass of the iteration is one launch over a sub-batch (solute =
// blockIdx.y), one batched cuFFT plan transforms all its site pairs, each
// solute converges on its own device state word (a finished solute's blocks
// idle), and the loop is the same captured graph.  Sub-batches run
// concurrently: each has its own child context and stream and is driven
// from its own host thread, so a sub-batch that has converged stops paying
// for the transforms of the others.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "rism3d_impl.h"

using namespace rism3d;

struct rism3d_ctx {
  Context c;
};

namespace {

// One batched solve with sub-batches of about kChunkPoints grid points.
int solve_batch_chunked(Context &p, int nmol, const int *natoms, const int *grids,
                        const double *boxes, const double *sig, const double *eps,
                        const double *q, const double *xyz, rism3d_result *results,
                        const std::vector<long long> &off, long long kChunkPoints) {
  // group by cell; a group larger than kChunkPoints grid points in all is
  // split into sub-batches that converge and finish on their own (a batch
  // moves in lock-step: its transforms run for every solute until the last
  // one converges) and run concurrently, each on its own stream.  For 256
  // solutes on 48^3 / 64^3 / 96^3 cells: one batch per cell 67 solves/s,
  // sub-batches of 2^25 / 2^22 / 2^20 / 2^18 points 72 / 79 / 86 / 84.
  std::map<std::pair<int, double>, std::vector<int>> cells;
  for (int m = 0; m < nmol; ++m) cells[{grids[m], boxes[m]}].push_back(m);
  std::map<std::pair<std::pair<int, double>, int>, std::vector<int>> groups;
  for (auto &kv : cells) {
    const long long n = (long long)kv.first.first * kv.first.first * kv.first.first;
    const int total = (int)kv.second.size();
    const int parts = (int)std::max<long long>(1, std::min<long long>(total, (n * total + kChunkPoints - 1) / kChunkPoints));
    for (int i = 0; i < total; ++i)        // even split, in input order
      groups[{kv.first, (int)((long long)i * parts / total)}].push_back(kv.second[i]);
  }
  // one child context per group, each on its own stream
  const long long call = ++p.batch_calls;
  std::vector<std::pair<Context *, const std::vector<int> *>> work;
  // 1. cached children with the shapes of this call's groups
  for (auto &kv : groups) {
    const int grid = kv.first.first.first;
    const double box = kv.first.first.second;
    const int nb = (int)kv.second.size();
    Context *ch = nullptr;                 // a cached child not yet taken by this call
    for (Context::Child &cc : p.children)
      if (!ch && cc.grid == grid && cc.box == box && cc.nb == nb && cc.last_call != call) {
        ch = cc.ctx;
        cc.last_call = call;
      }
    work.push_back({ch, &kv.second});
  }
  // 2. Children not used by this call stay cached for later calls with the
  // same shapes, up to a byte budget (RISM3D_BATCH_CACHE_BYTES, default
  // 4 GiB); beyond it the least recently used ones are freed -- before
  // this call allocates its new ones -- so callers whose batch composition
  // changes from call to call do not accumulate one context per composition.
  {
    size_t budget = 4ull << 30;
    if (const char *e = getenv("RISM3D_BATCH_CACHE_BYTES")) budget = (size_t)strtoull(e, nullptr, 10);
    for (;;) {
      size_t idle = 0;
      int lru = -1;
      for (size_t i = 0; i < p.children.size(); ++i) {
        const Context::Child &cc = p.children[i];
        if (cc.last_call == call) continue;
        idle += cc.bytes;
        if (lru < 0 || cc.last_call < p.children[lru].last_call) lru = (int)i;
      }
      if (idle <= budget || lru < 0) break;
      context_release(*p.children[lru].ctx);
      delete p.children[lru].ctx;
      p.children.erase(p.children.begin() + lru);
    }
  }
  // 3. new children for the groups without one
  for (auto &wk : work) {
    if (wk.first) continue;
    const int m0 = (*wk.second)[0];
    const int grid = grids[m0];
    const double box = boxes[m0];
    const int nb = (int)wk.second->size();
    size_t free0 = 0, free1 = 0, total = 0;
    cudaMemGetInfo(&free0, &total);
    rism3d_params cp = p.prm;
    cp.grid[0] = cp.grid[1] = cp.grid[2] = grid;
    cp.box[0] = cp.box[1] = cp.box[2] = box;
    cp.stream = nullptr;           // its own stream: groups run concurrently
    cp.verbose = 0;
    Context *ch = new Context;
    std::string err;
    int rc = context_init(*ch, &cp, nb, err);
    if (rc == RISM3D_OK)
      rc = context_set_solvent(*ch, p.natv, p.rho, p.qv, p.sigv, p.epsv, p.temper, p.xt,
                               p.ntab, p.xdr, p.xvv_host.data());
    if (rc != RISM3D_OK) {
      p.err = err.empty() ? ch->err : err;
      context_release(*ch);
      delete ch;
      return rc;
    }
    cudaMemGetInfo(&free1, &total);
    Context::Child cc;
    cc.grid = grid; cc.nb = nb; cc.box = box; cc.ctx = ch;
    cc.last_call = call;
    cc.bytes = free0 > free1 ? free0 - free1 : 0;
    p.children.push_back(cc);
    wk.first = ch;
  }
  // work queued on the caller's stream before this call comes first
  cudaEvent_t start = nullptr;
  if (!cuda_ok(p, cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "batch") ||
      !cuda_ok(p, cudaEventRecord(start, p.stream), "batch"))
    return RISM3D_CUDA_ERROR;
  // each group on its own host thread: potentials, solve, observables
  std::vector<int> rcs(work.size(), RISM3D_OK);
  auto run_group = [&](size_t gi) {
    Context *ch = work[gi].first;
    const std::vector<int> &mols = *work[gi].second;
    const int nb = (int)mols.size();
    cudaSetDevice(p.dev);
    cudaStreamWaitEvent(ch->stream, start, 0);
    std::vector<int> cnt(nb);
    std::vector<double> s, e, qq, r;
    for (int b = 0; b < nb; ++b) {
      const int m = mols[b];
      cnt[b] = natoms[m];
      s.insert(s.end(), sig + off[m], sig + off[m + 1]);
      e.insert(e.end(), eps + off[m], eps + off[m + 1]);
      qq.insert(qq.end(), q + off[m], q + off[m + 1]);
      r.insert(r.end(), xyz + 3 * off[m], xyz + 3 * off[m + 1]);
    }
    int rc = context_set_atoms(*ch, cnt, s.data(), e.data(), qq.data(), r.data());
    if (rc == RISM3D_OK) {
      ch->res = rism3d_result{};
      ch->bres.assign(nb, rism3d_result{});
      cudaEventRecord(ch->tm_iter.a, ch->stream);
      rc = run_solve(*ch, 0);
      cudaEventRecord(ch->tm_iter.b, ch->stream);
    }
    if (rc == RISM3D_OK) {
      cudaEventRecord(ch->tm_obs.a, ch->stream);
      rc = compute_observables(*ch);
      if (rc == RISM3D_OK) rc = compute_atom_integrals(*ch, false);
      cudaEventRecord(ch->tm_obs.b, ch->stream);
    }
    if (rc == RISM3D_OK && cudaStreamSynchronize(ch->stream) != cudaSuccess) {
      ch->err = "batch group: stream failed";
      rc = RISM3D_CUDA_ERROR;
    }
    rcs[gi] = rc;
  };
  std::vector<std::thread> threads;
  for (size_t gi = 1; gi < work.size(); ++gi) threads.emplace_back(run_group, gi);
  if (!work.empty()) run_group(0);
  for (std::thread &t : threads) t.join();
  cudaEventDestroy(start);
  int worst = RISM3D_OK;
  for (size_t gi = 0; gi < work.size(); ++gi) {
    Context *ch = work[gi].first;
    if (rcs[gi] != RISM3D_OK) {
      p.err = ch->err;
      return rcs[gi];
    }
    const std::vector<int> &mols = *work[gi].second;
    const int nb = (int)mols.size();
    float ms_s = 0, ms_i = 0, ms_o = 0;
    cudaEventElapsedTime(&ms_s, ch->tm_setup.a, ch->tm_setup.b);
    cudaEventElapsedTime(&ms_i, ch->tm_iter.a, ch->tm_iter.b);
    cudaEventElapsedTime(&ms_o, ch->tm_obs.a, ch->tm_obs.b);
    for (int b = 0; b < nb; ++b) {
      rism3d_result rr = nb == 1 ? ch->res : ch->bres[b];
      if (nb == 1) { rr.iterations = ch->res.iterations; rr.status = ch->res.status; }
      rr.natv = p.natv;
      rr.natom = natoms[mols[b]];
      rr.ms_setup = ms_s;                        // group totals
      rr.ms_iterate = ms_i;
      rr.ms_observe = ms_o;
      results[mols[b]] = rr;
      if (rr.status != RISM3D_OK && worst == RISM3D_OK) worst = rr.status;
    }
    p.launches += ch->launches;
    ch->launches = 0;
  }
  return worst;
}

}  // namespace

extern "C" int rism3d_solve_batch(rism3d_ctx *x, int nmol, const int *natoms, const int *grids,
                                  const double *boxes, const double *sig, const double *eps,
                                  const double *q, const double *xyz, rism3d_result *results) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &p = x->c;
  cudaSetDevice(p.dev);
  if (!p.have_solvent) { p.err = "set the solvent first"; return RISM3D_BAD_STATE; }
  if (nmol < 1 || !natoms || !grids || !boxes || !sig || !eps || !q || !xyz || !results) {
    p.err = "bad batch arguments";
    return RISM3D_BAD_INPUT;
  }
  std::vector<long long> off(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    if (natoms[m] < 1 || grids[m] < 4 || !(boxes[m] > 0)) {
      p.err = "bad batch entry " + std::to_string(m);
      return RISM3D_BAD_INPUT;
    }
    off[m + 1] = off[m] + natoms[m];
  }
  if (p.prm.batch_chunk_points > 0)
    return solve_batch_chunked(p, nmol, natoms, grids, boxes, sig, eps, q, xyz, results, off,
                               p.prm.batch_chunk_points);
  // Autotuned sub-batch size: the first call whose batch holds a given set
  // of cells runs the whole batch once per candidate size (wall time from
  // the call to the end of its last group), keeps the fastest for that set
  // and returns the last run's results (the sub-batch size does not change
  // any solute's equations, only which solutes share a launch).  Later calls
  // with the same set of cells use the cached size.
  std::string key;
  {
    std::map<std::pair<int, double>, int> cells;
    for (int m = 0; m < nmol; ++m) cells[{grids[m], boxes[m]}] += 1;
    for (auto &kv : cells)
      key += std::to_string(kv.first.first) + "/" + std::to_string(kv.first.second) + ";";
  }
  auto it = p.batch_tuned.find(key);
  if (it != p.batch_tuned.end())
    return solve_batch_chunked(p, nmol, natoms, grids, boxes, sig, eps, q, xyz, results, off,
                               it->second);
  static const long long kCandidates[] = {1LL << 18, 1LL << 19, 1LL << 20, 1LL << 21, 1LL << 22};
  long long best = 1LL << 20;
  double best_ms = 1e300;
  int rc = RISM3D_OK;
  for (long long cand : kCandidates) {
    if (!cuda_ok(p, cudaStreamSynchronize(p.stream), "batch tuning")) return RISM3D_CUDA_ERROR;
    const auto t0 = std::chrono::steady_clock::now();
    rc = solve_batch_chunked(p, nmol, natoms, grids, boxes, sig, eps, q, xyz, results, off, cand);
    if (rc == RISM3D_CUDA_ERROR || rc == RISM3D_CUFFT_ERROR || rc == RISM3D_BAD_INPUT ||
        rc == RISM3D_UNSUPPORTED_SHAPE || rc == RISM3D_BAD_STATE)
      return rc;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms < best_ms) { best_ms = ms; best = cand; }
  }
  p.batch_tuned[key] = best;
  if (best != kCandidates[sizeof(kCandidates) / sizeof(kCandidates[0]) - 1])
    rc = solve_batch_chunked(p, nmol, natoms, grids, boxes, sig, eps, q, xyz, results, off, best);
  return rc;
}
