// api.cpp - the C ABI: handle registries and the entry points of dnnf90.h
// and dnnf90_b200.h.
//
// The registry model is the reference's (lib/c_api_module.f90:38-62): 64
// slots per kind, handles are slot numbers > 0, a freed network slot
// advances a generation counter and every dependent object built for an
// earlier occupant is refused (-1).  Unlike the reference, no error stops
// the process: every failure is a negative return code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dnnf90.h"
#include "../../include/dnnf90_b200.h"
#include "engine.hpp"
#include "gemm_tc.hpp"

using namespace dnnf90;

namespace {

constexpr int MAXH = 64;
constexpr int QCAP = 8192;  // grad_point queue length before a flush

struct NetH {
  bool used = false;
  TableSet ts;
  int nlayer = 0;
  std::vector<int> dims;
  std::vector<double> w;  // flat layer layout
  uint64_t wver = 1;      // bumped on every host-side weight change
  int prec = PREC_F64;
  bool dt_ok = false;
  DevTables dt;
  DevNet dn;
};

struct WorkH {
  bool used = false;
  int nid = 0, gen = 0;
  Planes p;
  cudaStream_t st = nullptr;
  int chunk = 0;
  // planes kept by a keep=1 forward
  bool kept = false;
  const double *kept_x = nullptr;
  int kept_n = 0;
  uint64_t kept_ver = 0;
  // grad_point queue
  std::vector<double> qx, qs;
  int qn = 0, qgid = 0;
  double *dX = nullptr, *dS = nullptr;
  size_t dcap = 0;
};

struct GradH {
  bool used = false;
  int nid = 0, gen = 0;
  double *d = nullptr, *m = nullptr, *v = nullptr;
  int nw = 0;
};

struct TabH {
  bool used = false;
  TableSet ts;
};

struct RuleH {
  bool used = false;
  SeedRuleHost r;
  bool up = false;
  DevRule d;
};

// extended Kalman filter bound to a network (kalman_t, lib/kalman_module.f90:47-90)
struct KfH {
  bool used = false;
  int nid = 0, gen = 0;
  bool decoupled = false;
  std::vector<int> bsz, boff;
  KfDev d;
  cudaStream_t st = nullptr;
};

std::recursive_mutex g_mu;
TabH g_tab[MAXH + 1];
NetH g_net[MAXH + 1];
int g_gen[MAXH + 1];
WorkH g_wrk[MAXH + 1];
WorkH g_twk[MAXH + 1];
GradH g_grd[MAXH + 1];
RuleH g_rule[MAXH + 1];
KfH g_kf[MAXH + 1];
TableSet g_cur;
bool g_cur_ready = false;

template <typename T>
int free_slot(T *reg) {
  for (int i = 1; i <= MAXH; ++i)
    if (!reg[i].used) return i;
  set_error("every handle of this kind is in use (" + std::to_string(MAXH) + ")");
  return -1;
}

bool bad_net(int nid) { return nid < 1 || nid > MAXH || !g_net[nid].used; }

int ck(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return RC_OK;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;
}

int weight_count(const std::vector<int> &dims) {
  int n = 0;
  for (size_t l = 1; l < dims.size(); ++l) n += dims[l] * (dims[l - 1] + 1);
  return n;
}

// net_init contract checks (lib/net_module.f90:109-136)
int init_net(NetH &n, const TableSet &ts, int nlayer, const int *dims) {
  if (nlayer < 2) return RC_BAD_ARG;
  for (int l = 0; l < nlayer; ++l)
    if (dims[l] < 1) return RC_BAD_ARG;
  if (dims[0] != ts.d0) {
    set_error("input width does not match the table set d0");
    return RC_BAD_ARG;
  }
  n = NetH();
  n.used = true;
  n.ts = ts;
  n.nlayer = nlayer;
  n.dims.assign(dims, dims + nlayer);
  n.w.assign(weight_count(n.dims), 0.0);
  return RC_OK;
}

size_t layer_off(const NetH &n, int l) {  // 1-based l in 2..nlayer
  size_t o = 0;
  for (int ll = 2; ll < l; ++ll) o += (size_t)n.dims[ll - 1] * (n.dims[ll - 2] + 1);
  return o;
}

// device copies of the network's tables and weights, refreshed when stale
int net_device(NetH &n, cudaStream_t st) {
  int rc = device_ready();
  if (rc) return rc;
  if (!n.dt_ok) {
    if ((rc = upload_tables(n.ts, n.dt))) return rc;
    n.dt_ok = true;
  }
  if (n.dn.uploaded != n.wver) {
    DevNet &d = n.dn;
    if (!d.w64) {
      d.nlayer = n.nlayer;
      d.dims = n.dims;
      d.nw = (int)n.w.size();
      d.woff.assign(n.nlayer, 0);
      for (int l = 2; l <= n.nlayer; ++l) d.woff[l - 1] = layer_off(n, l);
      if ((rc = ck(cudaMalloc(&d.w64, n.w.size() * sizeof(double)), "cudaMalloc"))) return rc;
      if ((rc = ck(cudaMalloc(&d.w32, n.w.size() * sizeof(float)), "cudaMalloc"))) return rc;
      if ((rc = ck(cudaMalloc(&d.wpk, 2 * n.w.size() * sizeof(double)), "cudaMalloc"))) return rc;
    }
    if ((rc = ck(cudaMemcpyAsync(d.w64, n.w.data(), n.w.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, st), "weights H2D")))
      return rc;
    if ((rc = weights_to_f32(d.w64, d.w32, n.w.size(), st))) return rc;
    if ((rc = gemm_tc_prepare(&d, n.w.data(), st))) return rc;
    d.uploaded = n.wver;
  }
  return RC_OK;
}

int work_stream(WorkH &w) {
  if (!w.st) {
    int rc = ck(cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking), "stream");
    if (rc) return rc;
  }
  return RC_OK;
}

// planes for up to want points (bounded by a device memory budget)
// drops cached committee graphs that use a network or work space being freed
void comm_forget(int nid, int tid);

// device bytes of one point's planes on a network's work space
size_t plane_bytes_per_point(const NetH &n) {
  const size_t rsz = n.prec == PREC_F64 ? 8 : 4;
  size_t per = 0;
  int nmax = 0;
  for (int l = 1; l < n.nlayer; ++l) nmax = std::max(nmax, n.dims[l]);
  for (int l = 2; l < n.nlayer; ++l) per += 2 * (size_t)n.ts.na * n.dims[l - 1] * rsz;
  per += 3 * (size_t)n.ts.na * nmax * rsz;
  per += 2 * (size_t)n.ts.na * n.dims[n.nlayer - 1] * 8 + n.ts.d0 * 8 + 1024;
  per += (size_t)(n.ts.k + 2) * n.dims[1] * rsz;  // the first layer's s^(q)
  return per;
}

// points whose planes (every layer's T and h, the S / Sb / Tb scratch, the
// seeds and outputs: plane_bytes_per_point, so set by |A| = f(D0, K) and
// the widths) one chunk of work space w holds: at most 48 GiB, and at most
// half of what is free with this work space's own planes counted as free
// (so the cap does not grow by re-counting them on every call), and at most
// the chunk set by dnnf90_twork_set_chunk
int plane_cap(const WorkH &w, const NetH &n) {
  const size_t per = plane_bytes_per_point(n);
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  const size_t avail = freeb + (w.p.base ? w.p.bytes : 0);
  const size_t budget = std::min<size_t>((size_t)48 << 30, avail / 2);
  int cap = (int)std::min<size_t>(std::max<size_t>(1, budget / per), (size_t)INT32_MAX);
  if (w.chunk > 0) cap = std::min(cap, w.chunk);
  return cap;
}

int work_planes(WorkH &w, NetH &n, int want, bool exact) {
  const int cap = plane_cap(w, n);
  int need = std::min(want, cap);
  if (exact && want > cap) {
    set_error("the kept forward does not fit the device memory budget");
    return RC_NOMEM;
  }
  if (w.p.base && w.p.prec == n.prec && w.p.cap_pts >= need) return RC_OK;
  w.kept = false;
  return ensure_planes(n.dt, n.dn, n.prec, std::max(need, 1), w.p);
}

int grad_alloc(GradH &g) {
  if (g.d) return RC_OK;
  int rc = device_ready();
  if (rc) return rc;
  if ((rc = ck(cudaMalloc(&g.d, sizeof(double) * std::max(1, g.nw)), "cudaMalloc"))) return rc;
  return ck(cudaMemset(g.d, 0, sizeof(double) * std::max(1, g.nw)), "cudaMemset");
}

int rule_device(RuleH &r, const NetH &n) {
  const TableSet &ts = n.ts;
  for (int s : r.r.ind)
    if (s < 0 || s >= ts.na) {
      set_error("seed rule names a slot the table set does not carry");
      return RC_BAD_ARG;
    }
  for (size_t f = 0; f + 1 < r.r.sfac.size(); f += 2)
    if (r.r.sfac[f] >= n.dims[n.nlayer - 1] || r.r.sfac[f + 1] >= ts.na) {
      set_error("system seed rule names an output component or slot the network does not carry");
      return RC_BAD_ARG;
    }
  if (!r.up) {
    int rc = upload_rule(r.r, r.d);
    if (rc) return rc;
    r.up = true;
  }
  return RC_OK;
}

// Run the queued grad_point points of one training work space.
int flush_queue(int tid) {
  WorkH &w = g_twk[tid];
  if (!w.qn) return RC_OK;
  const int nid = w.nid, gid = w.qgid, np = w.qn;
  w.qn = 0;
  if (bad_net(nid) || g_gen[nid] != w.gen) return RC_OK;  // net gone: points dropped
  if (gid < 1 || gid > MAXH || !g_grd[gid].used) return RC_OK;
  NetH &n = g_net[nid];
  GradH &g = g_grd[gid];
  int rc;
  if ((rc = work_stream(w))) return rc;
  if ((rc = net_device(n, w.st))) return rc;
  if ((rc = grad_alloc(g))) return rc;
  const int nout = n.dims[n.nlayer - 1], na = n.ts.na, d0 = n.ts.d0;
  size_t need = (size_t)np * (d0 + (size_t)nout * na);
  if (w.dcap < need) {
    if (w.dX) cudaFree(w.dX);
    w.dX = nullptr;
    w.dcap = 0;
    if ((rc = ck(cudaMalloc(&w.dX, need * sizeof(double)), "cudaMalloc"))) return rc;
    w.dcap = need;
  }
  w.dS = w.dX + (size_t)np * d0;
  std::vector<double> sm((size_t)np * nout * na, 0.0);
  for (int p = 0; p < np; ++p)
    std::memcpy(&sm[(size_t)p * nout * na], &w.qs[(size_t)p * na], sizeof(double) * na);
  if ((rc = ck(cudaMemcpyAsync(w.dX, w.qx.data(), sizeof(double) * np * d0,
                               cudaMemcpyHostToDevice, w.st), "H2D")))
    return rc;
  if ((rc = ck(cudaMemcpyAsync(w.dS, sm.data(), sizeof(double) * sm.size(),
                               cudaMemcpyHostToDevice, w.st), "H2D")))
    return rc;
  if ((rc = work_planes(w, n, np, false))) return rc;
  DevRule given;
  given.kind = SEED_GIVEN;
  BatchArgs a;
  a.npts = np; a.X = w.dX; a.seeds = w.dS; a.grad = g.d; a.train = true; a.prec = n.prec;
  if ((rc = run_batch(n.dt, n.dn, given, w.p, a, w.st))) return rc;
  if ((rc = ck(cudaStreamSynchronize(w.st), "grad_point batch"))) return rc;
  return gemm_tc_flag(&n.dn, w.st);
}

int flush_for_grad(int gid) {
  int rc = RC_OK;
  for (int t = 1; t <= MAXH; ++t)
    if (g_twk[t].used && g_twk[t].qn && g_twk[t].qgid == gid) {
      int r = flush_queue(t);
      if (r && !rc) rc = r;
    }
  return rc;
}

int flush_for_net(int nid) {
  int rc = RC_OK;
  for (int t = 1; t <= MAXH; ++t)
    if (g_twk[t].used && g_twk[t].qn && g_twk[t].nid == nid) {
      int r = flush_queue(t);
      if (r && !rc) rc = r;
    }
  return rc;
}

void free_work(WorkH &w) {
  w.p.release();
  if (w.st) cudaStreamDestroy(w.st);
  if (w.dX) cudaFree(w.dX);
  w = WorkH();
}

bool table_args_ok(int d0, int k, int nseed, const int *seeds) {
  if (d0 < 1 || k < 1 || k > 15 || nseed < 0) return false;
  if (seeds)
    for (int i = 0; i < d0 * nseed; ++i)
      if (seeds[i] < 0 || seeds[i] > k) return false;
  return true;
}

// ---- nn_weight.dat (lib/net_module.f90:146-243) ----
struct Reader {
  std::vector<std::string> lines;
  size_t ln = 0;
  bool ok = true;
  // list-directed read of n values starting at a fresh record; the rest of
  // the last record is discarded
  std::vector<std::string> read(size_t n) {
    std::vector<std::string> out;
    while (out.size() < n) {
      if (ln >= lines.size()) { ok = false; return out; }
      std::istringstream is(lines[ln++]);
      std::string tok;
      while (out.size() < n && is >> tok) {
        if (tok[0] == '/' || tok[0] == '!') break;
        out.push_back(tok);
      }
    }
    return out;
  }
  void skip() {
    if (ln < lines.size()) ln++;
    else ok = false;
  }
};

double to_d(const std::string &s, bool &ok) {
  std::string t = s;
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) ok = false;
  return v;
}

int load_net(const char *fname, const TableSet &ts, int &out) {
  std::ifstream f(fname);
  if (!f) return RC_BAD_FILE;
  Reader r;
  std::string line;
  while (std::getline(f, line)) r.lines.push_back(line);
  r.skip();  // epoch
  auto h = r.read(2);
  bool ok = r.ok;
  if (!ok || h.size() < 2) return RC_BAD_FILE;
  int ifunc = (int)to_d(h[1], ok);
  if (!ok || ifunc < 0 || ifunc > 4) return RC_BAD_FILE;
  auto ao = r.read(2);
  if (!r.ok || ao.size() < 2 || (int)to_d(ao[1], ok) != 0) {
    set_error("the weight file has a nonlinear output layer");
    return RC_BAD_FILE;
  }
  auto nl = r.read(1);
  if (!r.ok) return RC_BAD_FILE;
  int nlayer = (int)to_d(nl[0], ok);
  if (!ok || nlayer < 2 || nlayer > 64) return RC_BAD_FILE;
  std::vector<int> dims(nlayer);
  for (int i = 0; i < nlayer; ++i) {
    auto v = r.read(1);
    if (!r.ok) return RC_BAD_FILE;
    dims[i] = (int)to_d(v[0], ok);
  }
  if (!ok) return RC_BAD_FILE;
  if (ts.iact != ifunc) {
    set_error("the weight file names another activation than the table set");
    return RC_BAD_FILE;
  }
  int id = free_slot(g_net);
  if (id < 0) return RC_BAD_ARG;
  NetH tmp;
  int rc = init_net(tmp, ts, nlayer, dims.data());
  if (rc) return rc;
  size_t p = 0;
  for (int l = 2; l <= nlayer; ++l) {
    r.skip();  // "#l=" header
    for (int j = 0; j < dims[l - 1]; ++j) {
      auto v = r.read(dims[l - 2] + 1);
      if (!r.ok) return RC_BAD_FILE;
      for (auto &s : v) tmp.w[p++] = to_d(s, ok);
    }
  }
  if (!ok) return RC_BAD_FILE;
  g_net[id] = std::move(tmp);
  out = id;
  return RC_OK;
}

int run_eval(int nid, WorkH &w, int npts, const double *x, double *tm,
             bool host) {
  NetH &n = g_net[nid];
  int rc;
  if ((rc = work_stream(w))) return rc;
  if ((rc = net_device(n, w.st))) return rc;
  const int na = n.ts.na, d0 = n.ts.d0, nout = n.dims[n.nlayer - 1];
  if ((rc = work_planes(w, n, npts, false))) return rc;
  DevRule none;
  const int cap = w.p.cap_pts;
  // host batches are staged through the plane buffers chunk by chunk
  for (int c0 = 0; c0 < npts; c0 += (host ? cap : npts)) {
    int np = host ? std::min(cap, npts - c0) : npts;
    BatchArgs a;
    a.npts = np;
    a.prec = n.prec;
    if (host) {
      if ((rc = ck(cudaMemcpyAsync(w.p.X, x + (size_t)c0 * d0, sizeof(double) * np * d0,
                                   cudaMemcpyHostToDevice, w.st), "H2D")))
        return rc;
      a.X = w.p.X;
      a.out = w.p.out;
    } else {
      a.X = x;
      a.out = tm;
    }
    if ((rc = run_batch(n.dt, n.dn, none, w.p, a, w.st))) return rc;
    if (host) {
      if ((rc = ck(cudaMemcpyAsync(tm + (size_t)c0 * na * nout, w.p.out,
                                   sizeof(double) * np * na * nout,
                                   cudaMemcpyDeviceToHost, w.st), "D2H")))
        return rc;
    }
  }
  if (host) {
    if ((rc = ck(cudaStreamSynchronize(w.st), "eval"))) return rc;
    return gemm_tc_flag(&n.dn, w.st);
  }
  return RC_OK;
}

// checks shared by the training entries: net, work space, accumulator
int check_train(int nid, int tid, int gid, bool need_gid) {
  if (bad_net(nid)) return RC_BAD_ARG;
  if (tid < 1 || tid > MAXH || !g_twk[tid].used) return RC_BAD_ARG;
  if (g_twk[tid].nid != nid || g_twk[tid].gen != g_gen[nid]) return RC_BAD_ARG;
  if (need_gid) {
    if (gid < 1 || gid > MAXH || !g_grd[gid].used) return RC_BAD_ARG;
    if (g_grd[gid].nid != nid || g_grd[gid].gen != g_gen[nid]) return RC_BAD_ARG;
  }
  return RC_OK;
}

// [npts][na][nout] -> [npts][nout][na] / output 1 only
void relayout(const double *src, double *dst, int npts, int na, int nout,
              bool first_only) {
  for (int p = 0; p < npts; ++p)
    for (int ia = 0; ia < na; ++ia) {
      const double *s = src + ((size_t)p * na + ia) * nout;
      if (first_only) dst[(size_t)p * na + ia] = s[0];
      else
        for (int o = 0; o < nout; ++o) dst[((size_t)p * nout + o) * na + ia] = s[o];
    }
}

// one training batch from host buffers (grad_batch, grad_rule_batch,
// jrow_batch).  kind SEED_GIVEN uses seed[npts][na] (output 1).
int host_train(int nid, int tid, int npts, const double *x, int kind,
               RuleH *rule, const double *seed, double *grad_dev, double *rows,
               double *loss, double *t, double *resid, const double *src = nullptr,
               double *tmall = nullptr) {
  NetH &n = g_net[nid];
  WorkH &w = g_twk[tid];
  int rc;
  if ((rc = flush_queue(tid))) return rc;
  if ((rc = work_stream(w))) return rc;
  if ((rc = net_device(n, w.st))) return rc;
  if (rule && (rc = rule_device(*rule, n))) return rc;
  if ((rc = work_planes(w, n, npts, false))) return rc;
  const int na = n.ts.na, d0 = n.ts.d0, nout = n.dims[n.nlayer - 1];
  const int cap = w.p.cap_pts;
  const int nw = (int)n.w.size();
  double *dseed = nullptr, *drows = nullptr, *dloss = nullptr;
  if (kind == SEED_GIVEN) {
    if ((rc = ck(cudaMalloc(&dseed, sizeof(double) * (size_t)cap * nout * na), "cudaMalloc"))) return rc;
  }
  if (rows) {
    if ((rc = ck(cudaMalloc(&drows, sizeof(double) * (size_t)cap * nw), "cudaMalloc"))) {
      if (dseed) cudaFree(dseed);
      return rc;
    }
  }
  if ((rc = ck(cudaMalloc(&dloss, sizeof(double)), "cudaMalloc"))) {
    if (dseed) cudaFree(dseed);
    if (drows) cudaFree(drows);
    return rc;
  }
  const int nres = rule ? rule->r.nres : 0;
  double *dsrc = nullptr;
  if (src && nres > 0 &&
      (rc = ck(cudaMalloc(&dsrc, sizeof(double) * (size_t)cap * nres), "cudaMalloc"))) {
    if (dseed) cudaFree(dseed);
    if (drows) cudaFree(drows);
    cudaFree(dloss);
    return rc;
  }
  cudaMemsetAsync(dloss, 0, sizeof(double), w.st);
  std::vector<double> sm, tbuf;
  for (int c0 = 0; c0 < npts && !rc; c0 += cap) {
    const int np = std::min(cap, npts - c0);
    rc = ck(cudaMemcpyAsync(w.p.X, x + (size_t)c0 * d0, sizeof(double) * np * d0,
                            cudaMemcpyHostToDevice, w.st), "H2D");
    if (rc) break;
    DevRule given;
    given.kind = SEED_GIVEN;
    if (kind == SEED_GIVEN) {
      sm.assign((size_t)np * nout * na, 0.0);
      for (int p = 0; p < np; ++p)
        std::memcpy(&sm[(size_t)p * nout * na], seed + (size_t)(c0 + p) * na, sizeof(double) * na);
      rc = ck(cudaMemcpyAsync(dseed, sm.data(), sizeof(double) * sm.size(),
                              cudaMemcpyHostToDevice, w.st), "H2D");
      if (rc) break;
    }
    if (dsrc) {
      rc = ck(cudaMemcpyAsync(dsrc, src + (size_t)c0 * nres, sizeof(double) * (size_t)np * nres,
                              cudaMemcpyHostToDevice, w.st), "H2D");
      if (rc) break;
    }
    BatchArgs a;
    a.npts = np; a.X = w.p.X; a.out = (t || resid || tmall) ? w.p.out : nullptr;
    a.src = dsrc;
    a.seeds = dseed; a.grad = rows ? nullptr : grad_dev; a.rows = drows;
    a.loss = dloss; a.train = true; a.prec = n.prec;
    rc = run_batch(n.dt, n.dn, rule ? rule->d : given, w.p, a, w.st);
    if (rc) break;
    if (rows) {
      rc = ck(cudaMemcpyAsync(rows + (size_t)c0 * nw, drows, sizeof(double) * (size_t)np * nw,
                              cudaMemcpyDeviceToHost, w.st), "D2H");
      if (rc) break;
    }
    if (t || resid || tmall) {
      tbuf.resize((size_t)np * na * nout);
      rc = ck(cudaMemcpyAsync(tbuf.data(), w.p.out, sizeof(double) * tbuf.size(),
                              cudaMemcpyDeviceToHost, w.st), "D2H");
      if (!rc) rc = ck(cudaStreamSynchronize(w.st), "sync");
      if (rc) break;
      if (tmall) relayout(tbuf.data(), tmall + (size_t)c0 * nout * na, np, na, nout, false);
      std::vector<double> t1((size_t)np * na);
      relayout(tbuf.data(), t1.data(), np, na, nout, true);
      if (t) std::memcpy(t + (size_t)c0 * na, t1.data(), sizeof(double) * t1.size());
      if (resid && rule) {
        const SeedRuleHost &r = rule->r;
        for (int p = 0; p < np; ++p) {
          const double *tp = &t1[(size_t)p * na];
          double R = 0.0;
          for (size_t k = 0; k < r.coeff.size(); ++k)
            R = r.nonlin[k] ? R + r.coeff[k] * tp[0] * tp[r.ind[k]] : R + r.coeff[k] * tp[r.ind[k]];
          resid[c0 + p] = R;
        }
      }
    }
  }
  double lv = 0.0;
  if (!rc) rc = ck(cudaMemcpyAsync(&lv, dloss, sizeof(double), cudaMemcpyDeviceToHost, w.st), "D2H");
  if (!rc) rc = ck(cudaStreamSynchronize(w.st), "train batch");
  if (!rc) rc = gemm_tc_flag(&n.dn, w.st);
  if (loss) *loss = lv;
  if (dseed) cudaFree(dseed);
  if (drows) cudaFree(drows);
  if (dsrc) cudaFree(dsrc);
  cudaFree(dloss);
  return rc;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------- tables
int dnnf90_tables_init_dense(int d0, int k) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!table_args_ok(d0, k, 0, nullptr)) return RC_BAD_ARG;
  TableSet ts;
  if (!build_tables(d0, k, 0, nullptr, ts).empty()) return RC_BAD_ARG;
  g_cur = std::move(ts);
  g_cur_ready = true;
  return RC_OK;
}

int dnnf90_tables_init_closure(int d0, int k, int nseed, const int *seeds) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!table_args_ok(d0, k, nseed, seeds)) return RC_BAD_ARG;
  TableSet ts;
  std::string e = build_tables(d0, k, nseed, seeds, ts);
  if (!e.empty()) {
    set_error(e);
    return RC_BAD_ARG;
  }
  g_cur = std::move(ts);
  g_cur_ready = true;
  return RC_OK;
}

int dnnf90_nderiv(void) { return g_cur_ready ? g_cur.na : 0; }

int dnnf90_alpha(int ia, int *a) {
  if (!g_cur_ready || ia < 1 || ia > g_cur.na) return RC_BAD_ARG;
  for (int i = 0; i < g_cur.d0; ++i) a[i] = g_cur.alpha[(size_t)(ia - 1) * g_cur.d0 + i];
  return RC_OK;
}

int dnnf90_tabset_dense(int d0, int k) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!table_args_ok(d0, k, 0, nullptr)) return RC_BAD_ARG;
  int id = free_slot(g_tab);
  if (id < 0) return RC_BAD_ARG;
  TableSet ts;
  if (!build_tables(d0, k, 0, nullptr, ts).empty()) return RC_BAD_ARG;
  g_cur = ts;  // the reference leaves the module tables holding the last set
  g_cur_ready = true;
  g_tab[id].ts = std::move(ts);
  g_tab[id].used = true;
  return id;
}

int dnnf90_tabset_closure(int d0, int k, int nseed, const int *seeds) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!table_args_ok(d0, k, nseed, seeds)) return RC_BAD_ARG;
  int id = free_slot(g_tab);
  if (id < 0) return RC_BAD_ARG;
  TableSet ts;
  std::string e = build_tables(d0, k, nseed, seeds, ts);
  if (!e.empty()) {
    set_error(e);
    return RC_BAD_ARG;
  }
  g_cur = ts;
  g_cur_ready = true;
  g_tab[id].ts = std::move(ts);
  g_tab[id].used = true;
  return id;
}

int dnnf90_tabset_nderiv(int tid) {
  if (tid < 1 || tid > MAXH || !g_tab[tid].used) return RC_BAD_ARG;
  return g_tab[tid].ts.na;
}

int dnnf90_tabset_free(int tid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (tid < 1 || tid > MAXH || !g_tab[tid].used) return RC_BAD_ARG;
  g_tab[tid].ts = TableSet();  // networks keep their own copy of the set
  g_tab[tid].used = false;
  return RC_OK;
}

int dnnf90_tabset_activation(int tid, int iact) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (tid < 1 || tid > MAXH || !g_tab[tid].used) return RC_BAD_ARG;
  if (iact < 0 || iact > 4) return RC_BAD_FILE;
  g_tab[tid].ts.iact = iact;
  return RC_OK;
}

// ------------------------------------------------------------- networks
int dnnf90_net_create(int nlayer, const int *dims) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_cur_ready || nlayer < 2 || !dims) return RC_BAD_ARG;
  int id = free_slot(g_net);
  if (id < 0) return RC_BAD_ARG;
  TableSet ts = g_cur;
  ts.iact = 0;
  NetH n;
  int rc = init_net(n, ts, nlayer, dims);
  if (rc) return rc;
  g_net[id] = std::move(n);
  return id;
}

int dnnf90_net_create_ts(int tid, int nlayer, const int *dims) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (nlayer < 2 || !dims) return RC_BAD_ARG;
  for (int l = 0; l < nlayer; ++l)
    if (dims[l] < 1) return RC_BAD_ARG;
  if (tid < 1 || tid > MAXH || !g_tab[tid].used) return RC_BAD_ARG;
  int id = free_slot(g_net);
  if (id < 0) return RC_BAD_ARG;
  NetH n;
  int rc = init_net(n, g_tab[tid].ts, nlayer, dims);
  if (rc) return rc;
  g_net[id] = std::move(n);
  return id;
}

int dnnf90_net_load(const char *filename) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!filename) return RC_BAD_ARG;
  std::ifstream f(filename);
  if (!f) return RC_BAD_FILE;
  if (!g_cur_ready) return RC_BAD_ARG;
  if (free_slot(g_net) < 0) return RC_BAD_ARG;
  TableSet ts = g_cur;
  ts.iact = 0;
  int id = 0;
  int rc = load_net(filename, ts, id);
  return rc ? rc : id;
}

int dnnf90_net_load_ts(int tid, const char *filename) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (tid < 1 || tid > MAXH || !g_tab[tid].used || !filename) return RC_BAD_ARG;
  std::ifstream f(filename);
  if (!f) return RC_BAD_FILE;
  if (free_slot(g_net) < 0) return RC_BAD_ARG;
  int id = 0;
  int rc = load_net(filename, g_tab[tid].ts, id);
  return rc ? rc : id;
}

int dnnf90_net_set_layer(int nid, int l, const double *wrow) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || l < 2 || l > g_net[nid].nlayer || !wrow) return RC_BAD_ARG;
  NetH &n = g_net[nid];
  flush_for_net(nid);  // queued points were added under the old weights
  size_t o = layer_off(n, l);
  std::memcpy(&n.w[o], wrow, sizeof(double) * n.dims[l - 1] * (n.dims[l - 2] + 1));
  n.wver++;
  return RC_OK;
}

int dnnf90_net_free(int nid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid)) return RC_BAD_ARG;
  comm_forget(nid, 0);
  NetH &n = g_net[nid];
  n.dt.release();
  n.dn.release();
  n = NetH();
  g_gen[nid]++;
  return RC_OK;
}

// ------------------------------------------------------------- evaluation
int dnnf90_work_create(int nid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid)) return RC_BAD_ARG;
  int id = free_slot(g_wrk);
  if (id < 0) return RC_BAD_ARG;
  g_wrk[id] = WorkH();
  g_wrk[id].used = true;
  g_wrk[id].nid = nid;
  g_wrk[id].gen = g_gen[nid];
  return id;
}

int dnnf90_work_free(int wid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (wid < 1 || wid > MAXH || !g_wrk[wid].used) return RC_BAD_ARG;
  free_work(g_wrk[wid]);
  return RC_OK;
}

static int check_eval(int nid, int wid) {
  if (bad_net(nid) || wid < 1 || wid > MAXH || !g_wrk[wid].used) return RC_BAD_ARG;
  if (g_wrk[wid].nid != nid || g_wrk[wid].gen != g_gen[nid]) return RC_BAD_ARG;
  return RC_OK;
}

int dnnf90_eval(int nid, int wid, const double *x, double *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_eval(nid, wid);
  if (rc) return rc;
  NetH &n = g_net[nid];
  const int na = n.ts.na, nout = n.dims[n.nlayer - 1];
  std::vector<double> tm((size_t)na * nout);
  if ((rc = run_eval(nid, g_wrk[wid], 1, x, tm.data(), true))) return rc;
  for (int ia = 0; ia < na; ++ia) t[ia] = tm[(size_t)ia * nout];
  return RC_OK;
}

int dnnf90_eval_batch(int nid, int wid, int npts, const double *x, double *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_eval(nid, wid);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && (!x || !t))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  const int na = n.ts.na, nout = n.dims[n.nlayer - 1];
  std::vector<double> tm((size_t)npts * na * nout);
  if ((rc = run_eval(nid, g_wrk[wid], npts, x, tm.data(), true))) return rc;
  relayout(tm.data(), t, npts, na, nout, true);
  return RC_OK;
}

int dnnf90_eval_batch_multi(int nid, int wid, int npts, const double *x, double *tmo) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_eval(nid, wid);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && (!x || !tmo))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  const int na = n.ts.na, nout = n.dims[n.nlayer - 1];
  std::vector<double> tm((size_t)npts * na * nout);
  if ((rc = run_eval(nid, g_wrk[wid], npts, x, tm.data(), true))) return rc;
  relayout(tm.data(), tmo, npts, na, nout, false);
  return RC_OK;
}

// ------------------------------------------------------------- training
int dnnf90_twork_create(int nid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid)) return RC_BAD_ARG;
  int id = free_slot(g_twk);
  if (id < 0) return RC_BAD_ARG;
  g_twk[id] = WorkH();
  g_twk[id].used = true;
  g_twk[id].nid = nid;
  g_twk[id].gen = g_gen[nid];
  return id;
}

int dnnf90_twork_free(int tid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (tid < 1 || tid > MAXH || !g_twk[tid].used) return RC_BAD_ARG;
  flush_queue(tid);
  comm_forget(0, tid);
  free_work(g_twk[tid]);
  return RC_OK;
}

int dnnf90_twork_set_chunk(int tid, int npts) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (tid < 1 || tid > MAXH || !g_twk[tid].used || npts < 0) return RC_BAD_ARG;
  g_twk[tid].chunk = npts;
  return RC_OK;
}

int dnnf90_grad_create(int nid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid)) return RC_BAD_ARG;
  int id = free_slot(g_grd);
  if (id < 0) return RC_BAD_ARG;
  g_grd[id] = GradH();
  g_grd[id].used = true;
  g_grd[id].nid = nid;
  g_grd[id].gen = g_gen[nid];
  g_grd[id].nw = (int)g_net[nid].w.size();
  return id;
}

int dnnf90_grad_free(int gid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (gid < 1 || gid > MAXH || !g_grd[gid].used) return RC_BAD_ARG;
  for (int t = 1; t <= MAXH; ++t)  // queued points of this accumulator die with it
    if (g_twk[t].used && g_twk[t].qgid == gid) g_twk[t].qn = 0;
  GradH &g = g_grd[gid];
  if (g.d) cudaFree(g.d);
  if (g.m) cudaFree(g.m);
  if (g.v) cudaFree(g.v);
  g = GradH();
  return RC_OK;
}

int dnnf90_grad_zero(int gid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (gid < 1 || gid > MAXH || !g_grd[gid].used) return RC_BAD_ARG;
  for (int t = 1; t <= MAXH; ++t)  // zeroing discards what was queued
    if (g_twk[t].used && g_twk[t].qgid == gid) g_twk[t].qn = 0;
  GradH &g = g_grd[gid];
  if (g.d) return ck(cudaMemset(g.d, 0, sizeof(double) * std::max(1, g.nw)), "grad_zero");
  return RC_OK;
}

int dnnf90_grad_point(int nid, int tid, const double *x, const double *seed, int gid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, gid, true);
  if (rc) return rc;
  if (!x || !seed) return RC_BAD_ARG;
  if ((rc = device_ready())) return rc;
  WorkH &w = g_twk[tid];
  NetH &n = g_net[nid];
  if (w.qn && w.qgid != gid)
    if ((rc = flush_queue(tid))) return rc;
  const int na = n.ts.na, d0 = n.ts.d0;
  if (w.qn == 0) {
    w.qx.resize((size_t)QCAP * d0);
    w.qs.resize((size_t)QCAP * na);
  }
  w.qgid = gid;
  std::memcpy(&w.qx[(size_t)w.qn * d0], x, sizeof(double) * d0);
  std::memcpy(&w.qs[(size_t)w.qn * na], seed, sizeof(double) * na);
  w.qn++;
  if (w.qn == QCAP) return flush_queue(tid);
  return RC_OK;
}

int dnnf90_adam_step(int nid, int gid, double eta, double beta1, double beta2,
                     double eps, int nbatch, int istep) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || gid < 1 || gid > MAXH || !g_grd[gid].used) return RC_BAD_ARG;
  if (g_grd[gid].nid != nid || g_grd[gid].gen != g_gen[nid]) return RC_BAD_ARG;
  int rc = flush_for_grad(gid);
  if (rc) return rc;
  NetH &n = g_net[nid];
  GradH &g = g_grd[gid];
  if ((rc = net_device(n, nullptr))) return rc;
  if ((rc = grad_alloc(g))) return rc;
  if (!g.m) {
    if ((rc = ck(cudaMalloc(&g.m, sizeof(double) * g.nw), "cudaMalloc"))) return rc;
    if ((rc = ck(cudaMalloc(&g.v, sizeof(double) * g.nw), "cudaMalloc"))) return rc;
    cudaMemset(g.m, 0, sizeof(double) * g.nw);
    cudaMemset(g.v, 0, sizeof(double) * g.nw);
  }
  if ((rc = adam_device(n.dn.w64, g.d, g.m, g.v, g.nw, eta, beta1, beta2, eps, nbatch,
                        istep, nullptr)))
    return rc;
  if ((rc = ck(cudaMemcpy(n.w.data(), n.dn.w64, sizeof(double) * n.w.size(),
                          cudaMemcpyDeviceToHost), "weights D2H")))
    return rc;
  n.wver++;  // the device FP32 / split copies follow on the next use
  return RC_OK;
}

// ------------------------------------------------------------- extensions
int dnnf90_net_set_precision(int nid, int prec) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || (prec != PREC_F64 && prec != PREC_SPLIT)) return RC_BAD_ARG;
  flush_for_net(nid);
  g_net[nid].prec = prec;
  return RC_OK;
}

int dnnf90_nweights(int nid) {
  if (bad_net(nid)) return RC_BAD_ARG;
  return (int)g_net[nid].w.size();
}

int dnnf90_net_get_layer(int nid, int l, double *wrow) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || l < 2 || l > g_net[nid].nlayer || !wrow) return RC_BAD_ARG;
  NetH &n = g_net[nid];
  std::memcpy(wrow, &n.w[layer_off(n, l)], sizeof(double) * n.dims[l - 1] * (n.dims[l - 2] + 1));
  return RC_OK;
}

int dnnf90_net_save(int nid, const char *filename) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || !filename) return RC_BAD_ARG;
  NetH &n = g_net[nid];
  FILE *f = std::fopen(filename, "w");
  if (!f) return RC_BAD_FILE;
  std::fprintf(f, "0\nfunc %d\nActivation_out 0\n%d\n", n.ts.iact, n.nlayer);
  for (int l = 0; l < n.nlayer; ++l) std::fprintf(f, "%d\n", n.dims[l]);
  size_t p = 0;
  for (int l = 2; l <= n.nlayer; ++l) {
    std::fprintf(f, " #l= %d\n", l);
    for (int j = 0; j < n.dims[l - 1]; ++j) {
      for (int i = 0; i <= n.dims[l - 2]; ++i) std::fprintf(f, "%25.16E", n.w[p++]);
      std::fprintf(f, "\n");
    }
  }
  std::fclose(f);
  return RC_OK;
}

int dnnf90_grad_batch(int nid, int tid, int npts, const double *x, const double *seed,
                      int gid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, gid, true);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && (!x || !seed))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  if ((rc = device_ready()) || (rc = grad_alloc(g_grd[gid]))) return rc;
  return host_train(nid, tid, npts, x, SEED_GIVEN, nullptr, seed, g_grd[gid].d, nullptr,
                    nullptr, nullptr, nullptr);
}

int dnnf90_seed_rule_create(int kind, int nterm, const double *coeff, const int *slot,
                            const int *nonlin, double fac) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (kind < SEED_HALFSQ || kind > SEED_JROW || nterm < 0) return RC_BAD_ARG;
  if (kind != SEED_HALFSQ && (nterm < 1 || !coeff || !slot)) return RC_BAD_ARG;
  int id = free_slot(g_rule);
  if (id < 0) return RC_BAD_ARG;
  RuleH r;
  r.used = true;
  r.r.kind = kind;
  r.r.fac = fac;
  for (int k = 0; k < nterm && kind != SEED_HALFSQ; ++k) {
    if (slot[k] < 1) return RC_BAD_ARG;
    r.r.coeff.push_back(coeff[k]);
    r.r.ind.push_back(slot[k] - 1);
    r.r.nonlin.push_back(nonlin ? (nonlin[k] ? 1 : 0) : 0);
  }
  g_rule[id] = std::move(r);
  return id;
}

int dnnf90_seed_rule_sys(int nres, int nterm, const int *res, const double *coeff,
                         const int *nfac, const int *comp, const int *slot, const double *wres,
                         double fac) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (nres < 1 || nres > SYS_MAXRES || nterm < 1 || !res || !coeff || !nfac || !comp || !slot) {
    set_error("dnnf90_seed_rule_sys: 1 <= nres <= " + std::to_string(SYS_MAXRES) +
              ", nterm >= 1 and every term array are required");
    return RC_BAD_ARG;
  }
  RuleH r;
  r.used = true;
  r.r.kind = SEED_SYS;
  r.r.fac = fac;
  r.r.nres = nres;
  int f = 0;
  for (int k = 0; k < nterm; ++k) {
    if (res[k] < 1 || res[k] > nres || nfac[k] < 1 || nfac[k] > SYS_MAXFAC) {
      set_error("dnnf90_seed_rule_sys: term " + std::to_string(k + 1) +
                ": residual outside 1..nres or factor count outside 1.." +
                std::to_string(SYS_MAXFAC));
      return RC_BAD_ARG;
    }
    r.r.sys.push_back(res[k] - 1);
    r.r.sys.push_back(nfac[k]);
    r.r.sys.push_back(f);
    r.r.coeff.push_back(coeff[k]);
    for (int m = 0; m < nfac[k]; ++m, ++f) {
      if (comp[f] < 1 || slot[f] < 1) {
        set_error("dnnf90_seed_rule_sys: components and slots are 1-based");
        return RC_BAD_ARG;
      }
      r.r.sfac.push_back(comp[f] - 1);
      r.r.sfac.push_back(slot[f] - 1);
    }
  }
  for (int i = 0; i < nres; ++i) r.r.wres.push_back(wres ? wres[i] : 1.0);
  int id = free_slot(g_rule);
  if (id < 0) return RC_BAD_ARG;
  g_rule[id] = std::move(r);
  return id;
}

int dnnf90_seed_rule_free(int rid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (rid < 1 || rid > MAXH || !g_rule[rid].used) return RC_BAD_ARG;
  g_rule[rid].d.release();
  g_rule[rid] = RuleH();
  return RC_OK;
}

static bool bad_rule(int rid) { return rid < 1 || rid > MAXH || !g_rule[rid].used; }

int dnnf90_grad_rule_batch(int nid, int tid, int npts, const double *x, int rid, int gid,
                           double *loss, double *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, gid, true);
  if (rc) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind == SEED_JROW) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && !x)) return RC_BAD_ARG;
  if (loss) *loss = 0.0;
  if (npts == 0) return RC_OK;
  if ((rc = device_ready()) || (rc = grad_alloc(g_grd[gid]))) return rc;
  return host_train(nid, tid, npts, x, g_rule[rid].r.kind, &g_rule[rid], nullptr,
                    g_grd[gid].d, nullptr, loss, t, nullptr);
}

int dnnf90_grad_sys_batch(int nid, int tid, int npts, const double *x, const double *src,
                          int rid, int gid, double *loss, double *tm) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, gid, true);
  if (rc) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind != SEED_SYS) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && !x)) return RC_BAD_ARG;
  if (loss) *loss = 0.0;
  if (npts == 0) return RC_OK;
  if ((rc = device_ready()) || (rc = grad_alloc(g_grd[gid]))) return rc;
  return host_train(nid, tid, npts, x, SEED_SYS, &g_rule[rid], nullptr, g_grd[gid].d, nullptr,
                    loss, nullptr, nullptr, src, tm);
}

int dnnf90_grad_value_batch(int nid, int tid, int npts, const double *x, const double *y,
                            double coef, int gid, double *loss) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, gid, true);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && (!x || !y))) return RC_BAD_ARG;
  if (g_net[nid].dims[g_net[nid].nlayer - 1] != 1) {
    set_error("dnnf90_grad_value_batch: the value fit is for a single output");
    return RC_BAD_ARG;
  }
  if (loss) *loss = 0.0;
  if (npts == 0) return RC_OK;
  if ((rc = device_ready()) || (rc = grad_alloc(g_grd[gid]))) return rc;
  // R = N(x) - y as a one-term system rule with source y: L = coef/2 R^2
  RuleH r;
  r.used = true;
  r.r.kind = SEED_SYS;
  r.r.fac = coef;
  r.r.nres = 1;
  r.r.sys = {0, 1, 0};
  r.r.sfac = {0, 0};
  r.r.coeff = {1.0};
  r.r.wres = {1.0};
  rc = host_train(nid, tid, npts, x, SEED_SYS, &r, nullptr, g_grd[gid].d, nullptr, loss, nullptr,
                  nullptr, y, nullptr);
  r.d.release();
  return rc;
}

int dnnf90_jrow_batch(int nid, int tid, int npts, const double *x, int rid, double *rows,
                      double *resid, double *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind != SEED_JROW) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!x || !rows))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  if ((rc = device_ready())) return rc;
  return host_train(nid, tid, npts, x, SEED_JROW, &g_rule[rid], nullptr, nullptr, rows,
                    nullptr, t, resid);
}

int dnnf90_grad_read(int gid, double *g) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (gid < 1 || gid > MAXH || !g_grd[gid].used || !g) return RC_BAD_ARG;
  int rc = flush_for_grad(gid);
  if (rc) return rc;
  GradH &gr = g_grd[gid];
  if (!gr.d) {
    std::memset(g, 0, sizeof(double) * gr.nw);
    return RC_OK;
  }
  return ck(cudaMemcpy(g, gr.d, sizeof(double) * gr.nw, cudaMemcpyDeviceToHost), "D2H");
}

static int ngd_host(int nid, int nrow, const double *rows, const double *b, int nb, double mu,
                    int prec, double *u, bool dual) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || nrow < 1 || nb < 1 || !rows || !b || !u) return RC_BAD_ARG;
  if (prec != PREC_F64 && prec != PREC_SPLIT) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  const int nw = (int)g_net[nid].w.size();
  double *dr = nullptr, *db = nullptr, *du = nullptr;
  if ((rc = ck(cudaMalloc(&dr, sizeof(double) * (size_t)nrow * nw), "cudaMalloc"))) return rc;
  if ((rc = ck(cudaMalloc(&db, sizeof(double) * nw * 2), "cudaMalloc"))) {
    cudaFree(dr);
    return rc;
  }
  du = db + nw;
  rc = ck(cudaMemcpy(dr, rows, sizeof(double) * (size_t)nrow * nw, cudaMemcpyHostToDevice), "H2D");
  if (!rc) rc = ck(cudaMemcpy(db, b, sizeof(double) * nw, cudaMemcpyHostToDevice), "H2D");
  if (!rc)
    rc = dual ? ngd_device_dual(dr, nrow, nw, db, nb, mu, du, prec, nullptr)
              : ngd_device(dr, nrow, nw, db, nb, mu, du, prec, nullptr);
  if (!rc) rc = ck(cudaMemcpy(u, du, sizeof(double) * nw, cudaMemcpyDeviceToHost), "D2H");
  cudaFree(dr);
  cudaFree(db);
  return rc;
}

int dnnf90_ngd_step(int nid, int nrow, const double *rows, const double *b, int nb,
                    double mu, int prec, double *u) {
  return ngd_host(nid, nrow, rows, b, nb, mu, prec, u, false);
}

int dnnf90_ngd_step_dual(int nid, int nrow, const double *rows, const double *b, int nb,
                         double mu, int prec, double *u) {
  return ngd_host(nid, nrow, rows, b, nb, mu, prec, u, true);
}

// ------------------------------------------------------------- device pointers
namespace {
// End of a device-pointer call on the split path: wait for the work on st and
// read the tensor-core GEMM's time-out flag, so that a GEMM that gave up is
// an error code rather than silently wrong planes.  Skipped while st is being
// captured into a graph (no synchronisation is allowed there).
int dev_finish(NetH &n, cudaStream_t st, int rc) {
  if (rc || n.prec != PREC_SPLIT) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return RC_OK;
  return gemm_tc_flag(&n.dn, st);
}
}  // namespace

int dnnf90_set_weights_dev(int nid, const double *w_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid) || !w_dev) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  NetH &n = g_net[nid];
  flush_for_net(nid);
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = ck(cudaMemcpyAsync(n.w.data(), w_dev, sizeof(double) * n.w.size(),
                               cudaMemcpyDeviceToHost, st), "weights D2H")))
    return rc;
  if ((rc = ck(cudaStreamSynchronize(st), "sync"))) return rc;
  n.wver++;
  return net_device(n, st);
}

int dnnf90_forward_dev(int nid, int tid, int npts, const double *x_dev, double *tm_dev,
                       int keep, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && !x_dev)) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  WorkH &w = g_twk[tid];
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = net_device(n, st))) return rc;
  if ((rc = work_planes(w, n, npts, keep != 0))) return rc;
  if (keep) {
    if ((rc = forward_keep(n.dt, n.dn, w.p, n.prec, npts, x_dev, tm_dev, st))) return rc;
    w.kept = true;
    w.kept_x = x_dev;
    w.kept_n = npts;
    w.kept_ver = n.wver;
    return dev_finish(n, st, RC_OK);
  }
  w.kept = false;
  DevRule none;
  BatchArgs a;
  a.npts = npts; a.X = x_dev; a.out = tm_dev; a.prec = n.prec;
  return dev_finish(n, st, run_batch(n.dt, n.dn, none, w.p, a, st));
}

int dnnf90_keep_fits(int nid, int tid, int npts, int *fits) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (npts < 0 || !fits) return RC_BAD_ARG;
  if ((rc = device_ready())) return rc;
  *fits = npts <= plane_cap(g_twk[tid], g_net[nid]) ? 1 : 0;
  return RC_OK;
}

int dnnf90_backward_dev(int nid, int tid, int npts, const double *x_dev,
                        const double *seedm_dev, double *grad_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (npts < 0 || (npts > 0 && (!x_dev || !seedm_dev || !grad_dev))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  WorkH &w = g_twk[tid];
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = net_device(n, st))) return rc;
  if (w.kept && w.kept_x == x_dev && w.kept_n == npts && w.kept_ver == n.wver &&
      w.p.prec == n.prec)
    return dev_finish(n, st,
                      adjoint_kept(n.dt, n.dn, w.p, n.prec, npts, x_dev, seedm_dev, grad_dev, st));
  // recompute mode: the forward runs again inside the adjoint
  if ((rc = work_planes(w, n, npts, false))) return rc;
  w.kept = false;
  DevRule given;
  given.kind = SEED_GIVEN;
  BatchArgs a;
  a.npts = npts; a.X = x_dev; a.seeds = seedm_dev; a.grad = grad_dev;
  a.train = true; a.prec = n.prec;
  return dev_finish(n, st, run_batch(n.dt, n.dn, given, w.p, a, st));
}

int dnnf90_grad_rule_dev(int nid, int tid, int npts, const double *x_dev, int rid,
                         double *grad_dev, double *loss_dev, double *tm_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind == SEED_JROW) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!x_dev || !grad_dev))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  WorkH &w = g_twk[tid];
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = net_device(n, st))) return rc;
  if ((rc = rule_device(g_rule[rid], n))) return rc;
  if ((rc = work_planes(w, n, npts, false))) return rc;
  w.kept = false;
  BatchArgs a;
  a.npts = npts; a.X = x_dev; a.out = tm_dev; a.grad = grad_dev; a.loss = loss_dev;
  a.train = true; a.prec = n.prec;
  return dev_finish(n, st, run_batch(n.dt, n.dn, g_rule[rid].d, w.p, a, st));
}

int dnnf90_jrow_dev(int nid, int tid, int npts, const double *x_dev, int rid,
                    double *rows_dev, double *tm_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = check_train(nid, tid, 0, false);
  if (rc) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind != SEED_JROW) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!x_dev || !rows_dev))) return RC_BAD_ARG;
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  WorkH &w = g_twk[tid];
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = net_device(n, st))) return rc;
  if ((rc = rule_device(g_rule[rid], n))) return rc;
  if ((rc = work_planes(w, n, npts, false))) return rc;
  w.kept = false;
  BatchArgs a;
  a.npts = npts; a.X = x_dev; a.out = tm_dev; a.rows = rows_dev;
  a.train = true; a.prec = n.prec;
  return dev_finish(n, st, run_batch(n.dt, n.dn, g_rule[rid].d, w.p, a, st));
}


// ------------------------------------------------------------- committee
extern "C++" {
namespace {
// One committee: its members, the streams and events of its graph, and the
// instantiated graph with the device addresses it baked in.
struct Committee {
  std::vector<int> nids, tids, rids, npts;
  std::vector<const double *> x;
  std::vector<double *> g;
  double *loss = nullptr;
  cudaStream_t caller = nullptr;
  cudaStream_t origin = nullptr;  // private stream the graph is captured on and
                                  // replayed on (the caller's may be the legacy
                                  // stream, which cannot be captured)
  cudaEvent_t ready = nullptr;    // caller's work before the step
  std::vector<cudaStream_t> st;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  std::vector<uintptr_t> sig;
  std::vector<double> work;
  int policy = -1;
  float ms = 0.f;
  ~Committee() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto s : st) if (s) cudaStreamDestroy(s);
    for (auto e : join) if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (ready) cudaEventDestroy(ready);
    if (origin) cudaStreamDestroy(origin);
  }
};
std::vector<std::unique_ptr<Committee>> g_comm;  // most recent last
int g_comm_policy = -1;
float g_comm_ms = 0.f;

// device addresses a captured graph depends on
std::vector<uintptr_t> comm_signature(const Committee &C) {
  std::vector<uintptr_t> v;
  for (size_t i = 0; i < C.nids.size(); ++i) {
    const NetH &n = g_net[C.nids[i]];
    const WorkH &w = g_twk[C.tids[i]];
    const RuleH &r = g_rule[C.rids[i]];
    v.push_back((uintptr_t)w.p.base);
    v.push_back((uintptr_t)w.p.cap_pts);
    v.push_back((uintptr_t)n.dn.w64);
    v.push_back((uintptr_t)n.dn.w32);
    v.push_back((uintptr_t)n.dn.tc);
    v.push_back((uintptr_t)n.dt.bp.id);
    v.push_back((uintptr_t)r.d.coeff);
    v.push_back((uintptr_t)n.prec);
  }
  return v;
}

// SMs member i may fill under a policy: 0 in proportion to its work,
// 1 in proportion to the square root of its work, 2 no cap
int comm_cap(const Committee &C, int i, int policy) {
  if (policy == 2) return 0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double tot = 0.0;
  for (double wv : C.work) tot += policy == 0 ? wv : std::sqrt(wv);
  const double mine = policy == 0 ? C.work[i] : std::sqrt(C.work[i]);
  return std::max(1, (int)std::lround(sms * mine / std::max(tot, 1e-300)));
}

// every member's zeroing and forward -> seed -> adjoint on its own stream,
// forked from and joined back into the origin stream
int comm_issue(Committee &C, int policy) {
  int rc = ck(cudaEventRecord(C.fork, C.origin), "committee fork");
  for (size_t i = 0; i < C.nids.size() && !rc; ++i) {
    NetH &n = g_net[C.nids[i]];
    WorkH &w = g_twk[C.tids[i]];
    RuleH &r = g_rule[C.rids[i]];
    cudaStream_t s = C.st[i];
    if ((rc = ck(cudaStreamWaitEvent(s, C.fork, 0), "committee wait"))) break;
    if ((rc = ck(cudaMemsetAsync(C.g[i], 0, sizeof(double) * n.w.size(), s), "memset"))) break;
    if ((rc = ck(cudaMemsetAsync(C.loss + i, 0, sizeof(double), s), "memset"))) break;
    set_grid_cap(comm_cap(C, (int)i, policy));
    BatchArgs a;
    a.npts = C.npts[i]; a.X = C.x[i]; a.grad = C.g[i]; a.loss = C.loss + i;
    a.train = true; a.prec = n.prec;
    rc = run_batch(n.dt, n.dn, r.d, w.p, a, s);
    set_grid_cap(0);
    if (rc) break;
    if ((rc = ck(cudaEventRecord(C.join[i], s), "committee join"))) break;
    rc = ck(cudaStreamWaitEvent(C.origin, C.join[i], 0), "committee wait");
  }
  return rc;
}

int comm_capture(Committee &C, int policy, cudaGraphExec_t *exec) {
  int rc = ck(cudaStreamBeginCapture(C.origin, cudaStreamCaptureModeRelaxed), "begin capture");
  if (rc) return rc;
  int rci = comm_issue(C, policy);
  cudaGraph_t graph = nullptr;
  rc = ck(cudaStreamEndCapture(C.origin, &graph), "end capture");
  if (rci) rc = rci;
  if (!rc) rc = ck(cudaGraphInstantiate(exec, graph, 0), "graph instantiate");
  if (graph) cudaGraphDestroy(graph);
  return rc;
}

// replays of an instantiated graph, the second one timed
int comm_time(Committee &C, cudaGraphExec_t exec, float *ms) {
  cudaEvent_t e0, e1;
  int rc = ck(cudaEventCreate(&e0), "event");
  if (rc) return rc;
  if ((rc = ck(cudaEventCreate(&e1), "event"))) { cudaEventDestroy(e0); return rc; }
  rc = ck(cudaGraphLaunch(exec, C.origin), "graph launch");
  if (!rc) rc = ck(cudaEventRecord(e0, C.origin), "event");
  if (!rc) rc = ck(cudaGraphLaunch(exec, C.origin), "graph launch");
  if (!rc) rc = ck(cudaEventRecord(e1, C.origin), "event");
  if (!rc) rc = ck(cudaEventSynchronize(e1), "graph replay");
  if (!rc) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// First call of a committee: work spaces under one memory budget, one
// untimed step outside any graph (it settles every allocation and the Bell
// kernels' variant choices), then one graph per SM-sharing policy, each
// replayed and timed; the fastest is kept.
int comm_build(Committee &C) {
  const int nn = (int)C.nids.size();
  C.exec = nullptr;
  if (C.st.empty()) {
    C.st.assign(nn, nullptr);
    C.join.assign(nn, nullptr);
    int rc = ck(cudaEventCreateWithFlags(&C.fork, cudaEventDisableTiming), "event");
    if (!rc) rc = ck(cudaEventCreateWithFlags(&C.ready, cudaEventDisableTiming), "event");
    if (!rc) rc = ck(cudaStreamCreateWithFlags(&C.origin, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < nn && !rc; ++i) {
      rc = ck(cudaStreamCreateWithFlags(&C.st[i], cudaStreamNonBlocking), "stream");
      if (!rc) rc = ck(cudaEventCreateWithFlags(&C.join[i], cudaEventDisableTiming), "event");
    }
    if (rc) return rc;
  }
  // memory: half of what is free (the members' own planes counted as free)
  // split in proportion to each member's need
  size_t freeb = 0, totb = 0, own = 0;
  cudaMemGetInfo(&freeb, &totb);
  double need = 0.0;
  for (int i = 0; i < nn; ++i) {
    own += g_twk[C.tids[i]].p.bytes;
    need += (double)C.npts[i] * plane_bytes_per_point(g_net[C.nids[i]]);
  }
  const double budget = 0.5 * (double)(freeb + own);
  const double scale = std::min(1.0, budget / std::max(need, 1.0));
  C.work.assign(nn, 0.0);
  for (int i = 0; i < nn; ++i) {
    NetH &n = g_net[C.nids[i]];
    WorkH &w = g_twk[C.tids[i]];
    w.chunk = std::max(std::min(C.npts[i], 64), (int)std::floor(C.npts[i] * scale));
    w.kept = false;
    int rc = work_planes(w, n, C.npts[i], false);
    if (rc) return rc;
    double per = 0.0;
    for (int l = 2; l < n.nlayer; ++l)
      per += (double)n.dims[l - 1] * ((double)n.ts.fq_ib.size() + n.ts.pair_ia.size() + 2.0 * n.ts.na);
    C.work[i] = per * C.npts[i];
  }
  int rc = ck(cudaEventRecord(C.ready, C.caller), "event");
  if (!rc) rc = ck(cudaStreamWaitEvent(C.origin, C.ready, 0), "wait");
  if (!rc) rc = comm_issue(C, 0);
  if (!rc) rc = ck(cudaStreamSynchronize(C.origin), "committee warm-up");
  if (rc) return rc;
  float best = 0.f;
  for (int pol = 0; pol < 3; ++pol) {
    cudaGraphExec_t ex = nullptr;
    if ((rc = comm_capture(C, pol, &ex))) return rc;
    float ms = 0.f;
    if ((rc = comm_time(C, ex, &ms))) {
      cudaGraphExecDestroy(ex);
      return rc;
    }
    if (!C.exec || ms < best) {
      if (C.exec) cudaGraphExecDestroy(C.exec);
      C.exec = ex;
      best = ms;
      C.policy = pol;
    } else {
      cudaGraphExecDestroy(ex);
    }
  }
  C.ms = best;
  C.sig = comm_signature(C);
  return RC_OK;
}

void comm_forget(int nid, int tid) {
  if (g_comm.empty()) return;
  cudaDeviceSynchronize();  // no replay of a graph may still run on these planes
  for (size_t i = 0; i < g_comm.size();) {
    const Committee &c = *g_comm[i];
    const bool hit = std::find(c.nids.begin(), c.nids.end(), nid) != c.nids.end() ||
                     std::find(c.tids.begin(), c.tids.end(), tid) != c.tids.end();
    if (hit) g_comm.erase(g_comm.begin() + i);
    else ++i;
  }
}
}  // namespace
}  // extern "C++"

int dnnf90_committee_step(int nnet, const int *nids, const int *tids, const int *rids,
                          const int *npts, const double *const *x_dev, double *const *grad_dev,
                          double *loss_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (nnet < 1 || nnet > MAXH || !nids || !tids || !rids || !npts || !x_dev || !grad_dev ||
      !loss_dev)
    return RC_BAD_ARG;
  for (int i = 0; i < nnet; ++i) {
    if (check_train(nids[i], tids[i], 0, false)) return RC_BAD_ARG;
    if (bad_rule(rids[i]) || g_rule[rids[i]].r.kind == SEED_JROW) return RC_BAD_ARG;
    if (npts[i] < 1 || !x_dev[i] || !grad_dev[i]) return RC_BAD_ARG;
    for (int k = 0; k < i; ++k)
      if (tids[k] == tids[i]) {
        set_error("committee members need distinct training work spaces");
        return RC_BAD_ARG;
      }
  }
  int rc = device_ready();
  if (rc) return rc;
  cudaStream_t caller = (cudaStream_t)stream;
  // weights, tables and rules on the device (rewritten in place when they
  // change, outside the graph)
  for (int i = 0; i < nnet; ++i) {
    NetH &n = g_net[nids[i]];
    flush_for_net(nids[i]);
    if ((rc = net_device(n, caller))) return rc;
    if ((rc = rule_device(g_rule[rids[i]], n))) return rc;
  }
  Committee *C = nullptr;
  for (auto &c : g_comm)
    if (c->caller == caller && c->loss == loss_dev &&
        c->nids == std::vector<int>(nids, nids + nnet) &&
        c->tids == std::vector<int>(tids, tids + nnet) &&
        c->rids == std::vector<int>(rids, rids + nnet) &&
        c->npts == std::vector<int>(npts, npts + nnet) &&
        c->x == std::vector<const double *>(x_dev, x_dev + nnet) &&
        c->g == std::vector<double *>(grad_dev, grad_dev + nnet))
      C = c.get();
  if (!C) {
    if (g_comm.size() >= 8) g_comm.erase(g_comm.begin());
    auto c = std::make_unique<Committee>();
    c->nids.assign(nids, nids + nnet);
    c->tids.assign(tids, tids + nnet);
    c->rids.assign(rids, rids + nnet);
    c->npts.assign(npts, npts + nnet);
    c->x.assign(x_dev, x_dev + nnet);
    c->g.assign(grad_dev, grad_dev + nnet);
    c->loss = loss_dev;
    c->caller = caller;
    C = c.get();
    g_comm.push_back(std::move(c));
  }
  if (!C->exec || C->sig != comm_signature(*C)) {
    if (C->exec) {
      cudaGraphExecDestroy(C->exec);
      C->exec = nullptr;
    }
    if ((rc = comm_build(*C))) return rc;
  }
  if ((rc = ck(cudaEventRecord(C->ready, caller), "event"))) return rc;
  if ((rc = ck(cudaStreamWaitEvent(C->origin, C->ready, 0), "wait"))) return rc;
  if ((rc = ck(cudaGraphLaunch(C->exec, C->origin), "graph launch"))) return rc;
  if ((rc = ck(cudaStreamSynchronize(C->origin), "committee step"))) return rc;
  for (int i = 0; i < nnet; ++i)
    if (g_net[nids[i]].prec == PREC_SPLIT && (rc = gemm_tc_flag(&g_net[nids[i]].dn, caller)))
      return rc;
  g_comm_policy = C->policy;
  g_comm_ms = C->ms;
  return RC_OK;
}

int dnnf90_tune_report(char *buf, int len) {
  static std::string pending;
  pending = tune_report();
  if (buf && len > 0) {
    std::strncpy(buf, pending.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)pending.size();
}

int dnnf90_tune_force(int which, int variant) {
  const int rc = which == 3 ? kf_force_path(variant) : tune_force(which, variant);
  if (rc)
    set_error("dnnf90_tune_force: which 0 or 1 with variant -1..7, 2 or 3 with -1..1");
  return rc;
}

int dnnf90_committee_info(int *policy, float *graph_ms) {
  if (policy) *policy = g_comm_policy;
  if (graph_ms) *graph_ms = g_comm_ms;
  return g_comm_policy >= 0 ? RC_OK : RC_BAD_ARG;
}

int dnnf90_ngd_gram_dev(int nrow, int nw, const double *rows_dev, int prec, double *G_dev,
                        void *stream) {
  if (nrow < 1 || nw < 1 || !rows_dev || !G_dev) return RC_BAD_ARG;
  if (prec != PREC_F64 && prec != PREC_SPLIT) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  return ngd_gram_device(rows_dev, nrow, nw, G_dev, prec, (cudaStream_t)stream);
}

int dnnf90_ngd_solve_dev(int nw, double *G_dev, const double *b_dev, int nb, double mu,
                         double *u_dev, void *stream) {
  if (nw < 1 || nb < 1 || !G_dev || !b_dev || !u_dev) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  return ngd_solve_device(G_dev, nw, b_dev, nb, mu, u_dev, (cudaStream_t)stream);
}

int dnnf90_ngd_step_dual_dev(int nrow, int nw, const double *rows_dev, const double *b_dev,
                             int nb, double mu, double *u_dev, void *stream) {
  if (nrow < 1 || nw < 1 || nb < 1 || !rows_dev || !b_dev || !u_dev) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  return ngd_device_dual(rows_dev, nrow, nw, b_dev, nb, mu, u_dev, PREC_F64,
                         (cudaStream_t)stream);
}

// ------------------------------------------------------------- Kalman filter
int dnnf90_kf_create(int nid, double p0, double lam_ini, double lam0, int decoupled, double q,
                     double gate) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (bad_net(nid)) return RC_BAD_ARG;
  // kf_init contract (lib/kalman_module.f90:118-127)
  if (!(p0 > 0.0)) {
    set_error("kf_create: p0 must be positive");
    return RC_BAD_ARG;
  }
  if (!(lam_ini > 0.0 && lam_ini <= 1.0 && lam0 > 0.0 && lam0 <= 1.0)) {
    set_error("kf_create: forgetting parameters must lie in (0,1]");
    return RC_BAD_ARG;
  }
  if (!(q >= 0.0) || !(gate >= 0.0)) {
    set_error("kf_create: process noise and gate must not be negative");
    return RC_BAD_ARG;
  }
  int rc = device_ready();
  if (rc) return rc;
  const int id = free_slot(g_kf);
  if (id < 0) return RC_BAD_ARG;
  const NetH &n = g_net[nid];
  KfH &k = g_kf[id];
  k = KfH();
  k.nid = nid;
  k.gen = g_gen[nid];
  k.decoupled = decoupled != 0;
  if (k.decoupled) {  // one block per neuron over (bias, fan-in), kf_block_map :172-189
    int m = 0;
    for (int l = 1; l < n.nlayer; ++l)
      for (int j = 0; j < n.dims[l]; ++j) {
        k.bsz.push_back(n.dims[l - 1] + 1);
        k.boff.push_back(m);
        m += n.dims[l - 1] + 1;
      }
  } else {
    k.bsz.push_back((int)n.w.size());
    k.boff.push_back(0);
  }
  if ((rc = kf_create(k.d, k.bsz, k.boff, p0, lam_ini, lam0, q, gate))) {
    k.d.release();
    k = KfH();
    return rc;
  }
  k.used = true;
  return id;
}

int dnnf90_kf_free(int kid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (kid < 1 || kid > MAXH || !g_kf[kid].used) return RC_BAD_ARG;
  KfH &k = g_kf[kid];
  if (k.st) cudaStreamSynchronize(k.st);
  k.d.release();
  if (k.st) cudaStreamDestroy(k.st);
  k = KfH();
  return RC_OK;
}

namespace {
int kf_check(int kid) {
  if (kid < 1 || kid > MAXH || !g_kf[kid].used) return RC_BAD_ARG;
  const KfH &k = g_kf[kid];
  if (bad_net(k.nid) || g_gen[k.nid] != k.gen) {
    set_error("kalman: the filter's network was freed");
    return RC_BAD_ARG;
  }
  return RC_OK;
}

// the filter's device staging area, grown to at least need bytes
int kf_stage(KfH &k, size_t need) {
  if (k.d.stage_bytes >= need) return RC_OK;
  cudaFree(k.d.stage);
  k.d.stage = nullptr;
  k.d.stage_bytes = 0;
  int rc = ck(cudaMalloc(&k.d.stage, need), "cudaMalloc");
  if (!rc) k.d.stage_bytes = need;
  return rc;
}

int kf_status_rc(const KfState &s) {
  if (!s.status) return RC_OK;
  if (s.status < 0) {
    set_error("kalman: a grid barrier of the one-launch update gave up waiting");
    return RC_DEVICE;
  }
  set_error("kalman: nonpositive innovation denominator at observation " +
            std::to_string(s.status) + "; the covariance has lost positive definiteness");
  return RC_BAD_ARG;
}
}  // namespace

int dnnf90_kf_update_rows(int kid, int nobs, const double *rows, const double *xi,
                          const double *scale) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = kf_check(kid);
  if (rc) return rc;
  if (nobs < 0 || (nobs > 0 && (!rows || !xi))) return RC_BAD_ARG;
  if (nobs == 0) return RC_OK;
  KfH &k = g_kf[kid];
  NetH &n = g_net[k.nid];
  flush_for_net(k.nid);  // queued points belong to the weights before the update
  if (!k.st && (rc = ck(cudaStreamCreateWithFlags(&k.st, cudaStreamNonBlocking), "stream")))
    return rc;
  const size_t nw = n.w.size();
  // rows staged in chunks of at most 256 MiB (DNNF90_KF_STAGE_KB overrides);
  // each chunk carries the first row of the next, whose products the
  // chunk's last tile pass forms
  size_t stage = 256u << 20;
  if (const char *e = std::getenv("DNNF90_KF_STAGE_KB")) stage = (size_t)std::max(1, std::atoi(e)) << 10;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(nobs, stage / (8 * nw)));
  const size_t need = ((size_t)(chunk + 1) * (nw + 2) + nw) * sizeof(double);
  if ((rc = kf_stage(k, need))) return rc;
  double *dw = k.d.stage, *dr = dw + nw, *dxi = dr + (size_t)(chunk + 1) * nw,
         *dsc = dxi + chunk + 1;
  if ((rc = ck(cudaMemcpyAsync(dw, n.w.data(), nw * 8, cudaMemcpyHostToDevice, k.st), "H2D")))
    return rc;
  for (int k0 = 0; k0 < nobs; k0 += chunk) {
    const int k1 = std::min(nobs, k0 + chunk);
    const int ncp = std::min(nobs, k1 + 1) - k0;  // rows staged, with the next chunk's first
    if ((rc = ck(cudaMemcpyAsync(dr, rows + (size_t)k0 * nw, (size_t)ncp * nw * 8,
                                 cudaMemcpyHostToDevice, k.st), "H2D")))
      return rc;
    if ((rc = ck(cudaMemcpyAsync(dxi, xi + k0, (size_t)ncp * 8, cudaMemcpyHostToDevice, k.st),
                 "H2D")))
      return rc;
    if (scale && (rc = ck(cudaMemcpyAsync(dsc, scale + k0, (size_t)ncp * 8,
                                          cudaMemcpyHostToDevice, k.st), "H2D")))
      return rc;
    if ((rc = kf_run(k.d, k1 - k0, dr, nw, dxi, scale ? dsc : nullptr, dw, k.st, k0,
                     k1 < nobs, k0 == 0)))
      return rc;
  }
  if ((rc = ck(cudaMemcpyAsync(n.w.data(), dw, nw * 8, cudaMemcpyDeviceToHost, k.st), "D2H")))
    return rc;
  KfState s;
  if ((rc = kf_state(k.d, &s, k.st))) return rc;
  n.wver++;
  return kf_status_rc(s);
}

int dnnf90_kf_update_rows_dev(int kid, int nobs, const double *rows_dev, const double *xi_dev,
                              const double *scale_dev, double *w_dev, void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = kf_check(kid);
  if (rc) return rc;
  if (nobs < 0 || (nobs > 0 && (!rows_dev || !xi_dev || !w_dev))) return RC_BAD_ARG;
  if (nobs == 0) return RC_OK;
  KfH &k = g_kf[kid];
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = kf_run(k.d, nobs, rows_dev, k.d.nw, xi_dev, scale_dev, w_dev, st, 0, false, true)))
    return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return RC_OK;
  KfState s;
  if ((rc = kf_state(k.d, &s, st))) return rc;
  return kf_status_rc(s);
}

namespace {
// the per-point filter pass: niter = 0 the plain update, >= 1 the iterated
// one with niter relinearisations per point
int kf_pass(int kid, int tid, int npts, const double *x, int rid, double rnoise, int niter) {
  int rc = kf_check(kid);
  if (rc) return rc;
  KfH &k = g_kf[kid];
  const int nid = k.nid;
  if ((rc = check_train(nid, tid, 0, false))) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind != SEED_JROW) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && !x)) return RC_BAD_ARG;
  if (!(rnoise > 0.0)) {  // kf_update_resid_multi :286-290
    set_error("kf_pass: observation noise must be > 0");
    return RC_BAD_ARG;
  }
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  if (n.prec != PREC_F64) {
    set_error("kf_pass: the per-point filter pass runs on the FP64 path (the filter moves "
              "the weights after every point)");
    return RC_UNSUPPORTED;
  }
  WorkH &w = g_twk[tid];
  RuleH &rule = g_rule[rid];
  if ((rc = flush_queue(tid))) return rc;
  flush_for_net(nid);
  if ((rc = work_stream(w))) return rc;
  if ((rc = net_device(n, w.st))) return rc;
  if ((rc = rule_device(rule, n))) return rc;
  if ((rc = work_planes(w, n, 1, false))) return rc;
  const int nw = (int)n.w.size(), d0 = n.ts.d0, nout = n.dims[n.nlayer - 1];
  const size_t need = ((size_t)npts * d0 + nw + 3) * sizeof(double);
  if ((rc = kf_stage(k, need))) return rc;
  double *drow = k.d.stage, *dxi = drow + nw, *dsc = dxi + 1, *dloss = dsc + 1,
         *dX = dloss + 1;
  const double sc = 1.0 / std::sqrt(rnoise);
  if ((rc = ck(cudaMemcpyAsync(dX, x, sizeof(double) * (size_t)npts * d0,
                               cudaMemcpyHostToDevice, w.st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(dsc, &sc, sizeof(double), cudaMemcpyHostToDevice, w.st), "H2D")))
    return rc;
  // per point: its row and residual at the current weights (the forward
  // and adjoint read the device weights the filter has just moved), then
  // the rank-one update of kf_update_resid (:252-275), xi = -R; or, iterated
  // (kf_iekf_begin / kf_iekf_iter :509-640), the prior stored and niter
  // relinearisations from it, the last one downdating the covariance
  BatchArgs a;
  a.npts = 1;
  a.out = w.p.out;
  a.rows = drow;
  a.loss = dloss;
  a.train = true;
  a.prec = PREC_F64;
  if (niter > 0 &&
      (rc = ck(cudaMemsetAsync(&k.d.st->status, 0, sizeof(int), w.st), "status reset")))
    return rc;
  for (int p = 0; p < npts && !rc; ++p) {
    a.X = dX + (size_t)p * d0;
    if (niter == 0) {
      if ((rc = run_batch(n.dt, n.dn, rule.d, w.p, a, w.st))) break;
      if ((rc = kf_resid_xi(rule.d, w.p.out, nout, dxi, w.st))) break;
      rc = kf_run(k.d, 1, drow, nw, dxi, dsc, n.dn.w64, w.st, p, false, true);
      continue;
    }
    if ((rc = ck(cudaMemcpyAsync(k.d.wprior, n.dn.w64, sizeof(double) * nw,
                                 cudaMemcpyDeviceToDevice, w.st), "D2D")))
      break;
    for (int it = 0; it < niter && !rc; ++it) {
      if ((rc = run_batch(n.dt, n.dn, rule.d, w.p, a, w.st))) break;
      if ((rc = kf_resid_xi(rule.d, w.p.out, nout, dxi, w.st, 1.0))) break;  // R itself
      rc = kf_iekf(k.d, drow, dxi, dsc, n.dn.w64, it == niter - 1, w.st, p, false);
    }
  }
  if (niter > 0) k.d.prior = false;  // the prior of the last point is not the caller's
  if (!rc) rc = ck(cudaMemcpyAsync(n.w.data(), n.dn.w64, sizeof(double) * nw,
                                   cudaMemcpyDeviceToHost, w.st), "D2H");
  KfState s;
  if (!rc) rc = kf_state(k.d, &s, w.st);
  n.wver++;  // the host copy now holds what the device computed
  return rc ? rc : kf_status_rc(s);
}
}  // namespace

int dnnf90_kf_pass(int kid, int tid, int npts, const double *x, int rid, double rnoise) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return kf_pass(kid, tid, npts, x, rid, rnoise, 0);
}

int dnnf90_kf_pass_iekf(int kid, int tid, int npts, const double *x, int rid, double rnoise,
                        int niter) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (niter < 1) {
    set_error("kf_pass_iekf: at least one iteration per point");
    return RC_BAD_ARG;
  }
  return kf_pass(kid, tid, npts, x, rid, rnoise, niter);
}

int dnnf90_kf_pass_sys(int kid, int tid, int npts, const double *x, const double *src, int rid,
                       const double *rnoise, int niter) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = kf_check(kid);
  if (rc) return rc;
  KfH &k = g_kf[kid];
  const int nid = k.nid;
  if ((rc = check_train(nid, tid, 0, false))) return rc;
  if (bad_rule(rid) || g_rule[rid].r.kind != SEED_SYS) return RC_BAD_ARG;
  if (npts < 0 || (npts > 0 && !x) || niter < 0) return RC_BAD_ARG;
  RuleH &rule = g_rule[rid];
  const int nres = rule.r.nres;
  std::vector<double> sc(nres, 1.0);
  for (int r = 0; r < nres && rnoise; ++r) {
    if (!(rnoise[r] > 0.0)) {  // kf_update_resid_multi :286-290
      set_error("kf_pass_sys: observation noise must be > 0");
      return RC_BAD_ARG;
    }
    sc[r] = 1.0 / std::sqrt(rnoise[r]);
  }
  if (npts == 0) return RC_OK;
  NetH &n = g_net[nid];
  if (n.prec != PREC_F64) {
    set_error("kf_pass_sys: the per-point filter pass runs on the FP64 path");
    return RC_UNSUPPORTED;
  }
  WorkH &w = g_twk[tid];
  if ((rc = flush_queue(tid))) return rc;
  flush_for_net(nid);
  if ((rc = work_stream(w))) return rc;
  if ((rc = net_device(n, w.st))) return rc;
  if ((rc = rule_device(rule, n))) return rc;
  if ((rc = work_planes(w, n, 1, false))) return rc;
  w.kept = false;  // the kept planes below belong to this pass
  const int nw = (int)n.w.size(), d0 = n.ts.d0, na = n.ts.na, nout = n.dims[n.nlayer - 1];
  const size_t need =
      ((size_t)nw + (size_t)nout * na + 1 + nres + (size_t)npts * (d0 + nres)) * sizeof(double);
  if ((rc = kf_stage(k, need))) return rc;
  double *drow = k.d.stage, *dseed = drow + nw, *dxi = dseed + (size_t)nout * na,
         *dsc = dxi + 1, *dX = dsc + nres, *dsrc = dX + (size_t)npts * d0;
  if ((rc = ck(cudaMemcpyAsync(dX, x, sizeof(double) * (size_t)npts * d0,
                               cudaMemcpyHostToDevice, w.st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(dsc, sc.data(), sizeof(double) * nres, cudaMemcpyHostToDevice,
                               w.st), "H2D")))
    return rc;
  if (src && (rc = ck(cudaMemcpyAsync(dsrc, src, sizeof(double) * (size_t)npts * nres,
                                      cudaMemcpyHostToDevice, w.st), "H2D")))
    return rc;
  if ((rc = ck(cudaMemsetAsync(&k.d.st->status, 0, sizeof(int), w.st), "status reset")))
    return rc;
  // per point and residual, at the current weights: the forward (planes
  // kept), R_ir and its seed, the adjoint into the row, then the update of
  // kf_update_resid_multi (xi = -R, scale 1/sqrt(rnoise_ir)); or, iterated,
  // niter relinearisations from the prior, the last one downdating
  auto observe = [&](int p, int r, double sign) {
    const double *xp = dX + (size_t)p * d0;
    int e = forward_keep(n.dt, n.dn, w.p, PREC_F64, 1, xp, w.p.out, w.st);
    if (!e) e = kf_sys_seed(rule.d, w.p.out, na, nout, src ? dsrc + (size_t)p * nres : nullptr,
                            r, dseed, dxi, sign, w.st);
    if (!e) e = ck(cudaMemsetAsync(drow, 0, sizeof(double) * nw, w.st), "memset");
    if (!e) e = adjoint_kept(n.dt, n.dn, w.p, PREC_F64, 1, xp, dseed, drow, w.st);
    return e;
  };
  for (int p = 0; p < npts && !rc; ++p)
    for (int r = 0; r < nres && !rc; ++r) {
      const int obs = p * nres + r;
      if (niter == 0) {
        if ((rc = observe(p, r, -1.0))) break;
        rc = kf_run(k.d, 1, drow, nw, dxi, dsc + r, n.dn.w64, w.st, obs == 0 ? 0 : obs, false,
                    true);
        continue;
      }
      if ((rc = ck(cudaMemcpyAsync(k.d.wprior, n.dn.w64, sizeof(double) * nw,
                                   cudaMemcpyDeviceToDevice, w.st), "D2D")))
        break;
      for (int it = 0; it < niter && !rc; ++it) {
        if ((rc = observe(p, r, 1.0))) break;
        rc = kf_iekf(k.d, drow, dxi, dsc + r, n.dn.w64, it == niter - 1, w.st, obs, false);
      }
    }
  if (niter > 0) k.d.prior = false;
  if (!rc) rc = ck(cudaMemcpyAsync(n.w.data(), n.dn.w64, sizeof(double) * nw,
                                   cudaMemcpyDeviceToHost, w.st), "D2H");
  KfState s;
  if (!rc) rc = kf_state(k.d, &s, w.st);
  n.wver++;
  return rc ? rc : kf_status_rc(s);
}

int dnnf90_kf_iekf_begin(int kid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = kf_check(kid);
  if (rc) return rc;
  KfH &k = g_kf[kid];
  const NetH &n = g_net[k.nid];
  if ((rc = ck(cudaMemcpy(k.d.wprior, n.w.data(), n.w.size() * 8, cudaMemcpyHostToDevice),
               "H2D")))
    return rc;
  k.d.prior = true;
  return RC_OK;
}

int dnnf90_kf_iekf_iter(int kid, const double *row, double resid, double rnoise, int final) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = kf_check(kid);
  if (rc) return rc;
  if (!row) return RC_BAD_ARG;
  KfH &k = g_kf[kid];
  if (!k.d.prior) {
    set_error("kf_iekf_iter: no prior (call dnnf90_kf_iekf_begin first)");
    return RC_BAD_ARG;
  }
  if (!(rnoise > 0.0)) {  // kf_iekf_iter :547-550
    set_error("kf_iekf_iter: observation noise must be > 0");
    return RC_BAD_ARG;
  }
  NetH &n = g_net[k.nid];
  flush_for_net(k.nid);
  if (!k.st && (rc = ck(cudaStreamCreateWithFlags(&k.st, cudaStreamNonBlocking), "stream")))
    return rc;
  const size_t nw = n.w.size();
  const size_t need = (2 * nw + 2) * sizeof(double);
  if ((rc = kf_stage(k, need))) return rc;
  double *dw = k.d.stage, *dr = dw + nw, *dsc = dr + nw;
  const double sc[2] = {1.0 / std::sqrt(rnoise), resid};
  if ((rc = ck(cudaMemcpyAsync(dw, n.w.data(), nw * 8, cudaMemcpyHostToDevice, k.st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(dr, row, nw * 8, cudaMemcpyHostToDevice, k.st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(dsc, sc, 16, cudaMemcpyHostToDevice, k.st), "H2D")))
    return rc;
  if ((rc = kf_iekf(k.d, dr, dsc + 1, dsc, dw, final != 0, k.st))) return rc;
  if ((rc = ck(cudaMemcpyAsync(n.w.data(), dw, nw * 8, cudaMemcpyDeviceToHost, k.st), "D2H")))
    return rc;
  KfState s;
  if ((rc = kf_state(k.d, &s, k.st))) return rc;
  n.wver++;
  return kf_status_rc(s);
}

int dnnf90_kf_read(int kid, double *lam, int *ngated, double *P) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (kid < 1 || kid > MAXH || !g_kf[kid].used) return RC_BAD_ARG;
  KfH &k = g_kf[kid];
  if (k.st) cudaStreamSynchronize(k.st);
  KfState s;
  int rc = kf_state(k.d, &s, nullptr);
  if (rc) return rc;
  if (lam) *lam = s.lam;
  if (ngated) *ngated = s.ngated;
  if (P) rc = kf_read_cov(k.d, k.bsz, k.boff, !k.decoupled, P, nullptr);
  return rc;
}

int dnnf90_kf_status(int kid) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (kid < 1 || kid > MAXH || !g_kf[kid].used) return RC_BAD_ARG;
  KfH &k = g_kf[kid];
  if (k.st) cudaStreamSynchronize(k.st);
  KfState s;
  const int rc = kf_state(k.d, &s, nullptr);
  if (rc) return rc;
  return s.status < 0 ? RC_DEVICE : s.status;
}

int dnnf90_ngd_step_noalloc(int nrow, int nw, const double *rows_dev, const double *b_dev,
                            int nb, double mu, double *u_dev, void *stream) {
  if (nrow < 1 || nw < 1 || nb < 1 || !rows_dev || !b_dev || !u_dev) return RC_BAD_ARG;
  int rc = device_ready();
  if (rc) return rc;
  return ngd_device_noalloc(rows_dev, nrow, nw, b_dev, nb, mu, u_dev, (cudaStream_t)stream);
}

const char *dnnf90_last_error(void) { return last_error(); }

long long dnnf90_launch_count(void) { return launch_count(); }

int dnnf90_profile_enable(int on) {
  profile_enable(on != 0);
  return RC_OK;
}

int dnnf90_profile_read(char *buf, int len) {
  // a call without a buffer collects the records and reports the length;
  // the next call with a buffer hands the same text out
  static std::string pending;
  static bool have = false;
  if (!have) {
    pending = profile_read();
    have = true;
  }
  const int need = (int)pending.size() + 1;
  if (!buf || len <= 0) return need;
  std::snprintf(buf, (size_t)len, "%s", pending.c_str());
  pending.clear();
  have = false;
  return need;
}

int dnnf90_device_available(void) { return device_ready() == RC_OK ? 1 : 0; }

}  // extern "C"
