// capi_dd.cu -- the time-slab domain decomposition behind the bqcdg_dd_* entry
// points of include/bqcdg.h: one context per slab (a lattice of Lt / nranks
// time slices), the face exchange before every stencil pass, the global sums
// of the CG, and two ways for the slabs to talk:
//
//   local  all slabs of the lattice in this process on one device; a face is
//          packed straight into the neighbour slab's ghost buffer and a global
//          sum adds the slabs' partial sums on the host in rank order.  This
//          is how the decomposition runs (and is tested) on one GPU.
//   nccl   one slab per process and GPU; faces go by ncclSend / ncclRecv into
//          the ghost buffers and global sums by ncclAllReduce, all on the
//          slab's stream.  libnccl.so.2 is opened at run time (the one a
//          process such as PyTorch has loaded already, if any).
//
// Every stencil pass overlaps the exchange with the slab's interior: the
// faces are packed and sent on an exchange stream (xstream) as soon as the
// input field is ready, the interior slices 1 .. Lt_loc-2, which read no
// ghost, run meanwhile on the compute stream, and the two boundary slices
// run after the exchange (an event).  Each site's arithmetic is that of one
// whole-slab launch, so the split changes no result.
//
// The reference does the same over MPI: project to half spinors
// (d/D21.F90:53), exchange the faces (xbound, comm/xbound_mpi.F90:418-461),
// compute (d/D21.F90:58-72), and global_sum the CG scalars (cg.F90:91,97,109).
#include <dlfcn.h>
#include <nccl.h>

#include "ctx.cuh"
#include "decomp.cuh"

namespace bqcdg {
void launch_dd_pack(const Geom& g, const DdGeom& d, bool dag, const double2* in, double2* to_prev, double2* to_next,
                    cudaStream_t s);
void launch_dd_pack_links(const Geom& g, const DdGeom& d, const double2* gauge, double2* to_next, cudaStream_t s);
void launch_dd_dslash(const Geom& g, const DdGeom& d, int e, bool dag, double2* out, const double2* in,
                      const double2* gauge, cudaStream_t s);
// part: 0 the whole slab, 1 its interior slices, 2 its boundary slices (dd_part_sites)
void launch_dd_pass1(const Geom& g, const DdGeom& d, bool dag, double2* out, const double2* in, const double2* gauge,
                     const double2* ainv, const OpParams& op, cudaStream_t s, int part);
void launch_dd_pass2(const Geom& g, const DdGeom& d, bool dag, double2* out, const double2* t, const double2* in,
                     const double2* gauge, const double2* aee, const OpParams& op, cudaStream_t s, int part);
// int16 slab passes (decomp16.cu); the second halves return the number of
// blocks whose partials they stored from slot0 on
void launch_dd16_pack(const Geom& g, const DdGeom& d, bool dag, SpinorPtr in, float2* to_prev, float2* to_next,
                      cudaStream_t s);
void launch_dd16_pass1(const Geom& g, const DdGeom& d, bool dag, int part, SpinorPtr out, SpinorPtr in,
                       const void* gauge, CloverPtr ainv, const OpParams& op, const CgScalars* cg, cudaStream_t s);
int launch_dd16_pass2(const Geom& g, const DdGeom& d, bool dag, int part, SpinorPtr out, SpinorPtr t, SpinorPtr x,
                      const void* gauge, CloverPtr aee, const OpParams& op, double* partial, int slot0,
                      const CgScalars* cg, cudaStream_t s);
int launch_dd16_pass4(const Geom& g, const DdGeom& d, int part, SpinorPtr t, SpinorPtr q, const void* gauge,
                      CloverPtr aee, const OpParams& op, SpinorPtr r, double* partial, int slot0, const CgScalars* cg,
                      cudaStream_t s);
void launch_dd_total(const DdPartials& parts, int nslabs, int nsb, CgScalars* cg, double* out, int mode,
                     cudaStream_t s);
void launch_dd_apply(const double* tot, CgScalars* cg, int mode, cudaStream_t s);
}  // namespace bqcdg

using namespace bqcdg_host;

namespace {

// the NCCL calls this file makes, resolved from libnccl.so.2 at run time
struct NcclApi {
  void* lib = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*groupStart)() = nullptr;
  ncclResult_t (*groupEnd)() = nullptr;
  ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*allReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  bool load() {
    if (lib) return true;
    lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) return false;
    getUniqueId = (decltype(getUniqueId))dlsym(lib, "ncclGetUniqueId");
    commInitRank = (decltype(commInitRank))dlsym(lib, "ncclCommInitRank");
    commDestroy = (decltype(commDestroy))dlsym(lib, "ncclCommDestroy");
    groupStart = (decltype(groupStart))dlsym(lib, "ncclGroupStart");
    groupEnd = (decltype(groupEnd))dlsym(lib, "ncclGroupEnd");
    send = (decltype(send))dlsym(lib, "ncclSend");
    recv = (decltype(recv))dlsym(lib, "ncclRecv");
    allReduce = (decltype(allReduce))dlsym(lib, "ncclAllReduce");
    return getUniqueId && commInitRank && commDestroy && groupStart && groupEnd && send && recv && allReduce;
  }
};
NcclApi g_nccl;

// device buffers of one slab for the exchange
struct SlabBufs {
  double2* ghost_fwd = nullptr;   // [6][V3h]
  double2* ghost_bwd = nullptr;   // [6][V3h]
  double2* ghost_link = nullptr;  // [2][9][V3h]
  double2* send_prev = nullptr;   // nccl: [6][V3h] for rank-1
  double2* send_next = nullptr;   // nccl: [6][V3h] for rank+1
  double2* send_links = nullptr;  // nccl: [2][9][V3h] for rank+1
};

}  // namespace

struct bqcdg_dd {
  bool nccl = false;
  int nranks = 1, rank0 = 0;  // rank of slabs[0]
  int L[4] = {0, 0, 0, 0}, bc[4] = {0, 0, 0, 0};
  int Lt_loc = 0, V3h = 0, volh_loc = 0;
  std::vector<bqcdg_ctx*> slabs;
  std::vector<SlabBufs> bufs;
  cudaStream_t stream = nullptr;  // every slab computes on the first slab's stream
  cudaStream_t xstream = nullptr; // face packing and exchange
  cudaEvent_t ev_ready = nullptr; // on stream: the field to exchange is written
  cudaEvent_t ev_done = nullptr;  // on xstream: the ghosts are filled
  ncclComm_t comm = nullptr;
  double* dsum = nullptr;         // nccl: device scalars of the global sums
  double* dtot = nullptr;         // the mixed solver's reduction total
  std::vector<double> hsum;

  int nslabs() const { return (int)slabs.size(); }
  DdGeom geom(int s) const {
    DdGeom d{};
    d.nranks = nranks;
    d.rank = rank0 + s;
    d.Lt_glob = L[3];
    d.t0 = (rank0 + s) * Lt_loc;
    d.V3h = V3h;
    d.bct = bc[3];
    d.ghost_fwd = bufs[s].ghost_fwd;
    d.ghost_bwd = bufs[s].ghost_bwd;
    d.ghost_link = bufs[s].ghost_link;
    return d;
  }
};

namespace {

int dd_check(bqcdg_dd* dd) { return dd && !dd->slabs.empty() ? BQCDG_OK : BQCDG_EINVAL; }

// the two timing events of a solve, released on every return path
struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t create() {
    cudaError_t e = cudaEventCreate(&e0);
    return e == cudaSuccess ? cudaEventCreate(&e1) : e;
  }
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// the faces of field f[s] of every slab, for passes with (dag) or without
// the dagger, into the ghost buffers of their neighbours: queued on xstream
// after everything queued so far on the compute stream (which includes the
// last reads of the ghosts this overwrites)
int dd_exchange(bqcdg_dd* dd, const std::vector<double2*>& f, bool dag) {
  const int n = dd->nslabs();
  CK(cudaEventRecord(dd->ev_ready, dd->stream));
  CK(cudaStreamWaitEvent(dd->xstream, dd->ev_ready, 0));
  if (!dd->nccl) {
    for (int s = 0; s < n; s++) {
      const int prev = (s + n - 1) % n, next = (s + 1) % n;
      launch_dd_pack(dd->slabs[s]->g, dd->geom(s), dag, f[s], dd->bufs[prev].ghost_fwd, dd->bufs[next].ghost_bwd,
                     dd->xstream);
    }
    CKL();
  } else {
    SlabBufs& b = dd->bufs[0];
    launch_dd_pack(dd->slabs[0]->g, dd->geom(0), dag, f[0], b.send_prev, b.send_next, dd->xstream);
    CKL();
    const int r = dd->rank0, prev = (r + dd->nranks - 1) % dd->nranks, next = (r + 1) % dd->nranks;
    const size_t cnt = (size_t)6 * dd->V3h * 2;  // doubles per face
    if (g_nccl.groupStart() != ncclSuccess) return BQCDG_ECUDA;
    ncclResult_t e = g_nccl.send(b.send_prev, cnt, ncclDouble, prev, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.recv(b.ghost_fwd, cnt, ncclDouble, next, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.send(b.send_next, cnt, ncclDouble, next, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.recv(b.ghost_bwd, cnt, ncclDouble, prev, dd->comm, dd->xstream);
    if (g_nccl.groupEnd() != ncclSuccess || e != ncclSuccess) return BQCDG_ECUDA;
  }
  return BQCDG_OK;
}
// the boundary launches that read the ghosts are queued on xstream after the
// exchange; then dd_exchange_done marks the end of the exchange stream's
// work, and dd_wait_exchange joins it into the compute stream
int dd_exchange_done(bqcdg_dd* dd) {
  CK(cudaEventRecord(dd->ev_done, dd->xstream));
  return BQCDG_OK;
}
int dd_wait_exchange(bqcdg_dd* dd) {
  CK(cudaStreamWaitEvent(dd->stream, dd->ev_done, 0));
  return BQCDG_OK;
}

// dd_exchange for an int16 field: FP32 faces (half the bytes of the FP64
// ones) in the same ghost and send buffers
int dd_exchange16(bqcdg_dd* dd, const std::vector<SpinorPtr>& f, bool dag) {
  const int n = dd->nslabs();
  CK(cudaEventRecord(dd->ev_ready, dd->stream));
  CK(cudaStreamWaitEvent(dd->xstream, dd->ev_ready, 0));
  if (!dd->nccl) {
    for (int s = 0; s < n; s++) {
      const int prev = (s + n - 1) % n, next = (s + 1) % n;
      launch_dd16_pack(dd->slabs[s]->g, dd->geom(s), dag, f[s], (float2*)dd->bufs[prev].ghost_fwd,
                       (float2*)dd->bufs[next].ghost_bwd, dd->xstream);
    }
    CKL();
  } else {
    SlabBufs& b = dd->bufs[0];
    launch_dd16_pack(dd->slabs[0]->g, dd->geom(0), dag, f[0], (float2*)b.send_prev, (float2*)b.send_next,
                     dd->xstream);
    CKL();
    const int r = dd->rank0, prev = (r + dd->nranks - 1) % dd->nranks, next = (r + 1) % dd->nranks;
    const size_t cnt = (size_t)6 * dd->V3h * 2;  // floats per face
    if (g_nccl.groupStart() != ncclSuccess) return BQCDG_ECUDA;
    ncclResult_t e = g_nccl.send(b.send_prev, cnt, ncclFloat, prev, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.recv(b.ghost_fwd, cnt, ncclFloat, next, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.send(b.send_next, cnt, ncclFloat, next, dd->comm, dd->xstream);
    if (e == ncclSuccess) e = g_nccl.recv(b.ghost_bwd, cnt, ncclFloat, prev, dd->comm, dd->xstream);
    if (g_nccl.groupEnd() != ncclSuccess || e != ncclSuccess) return BQCDG_ECUDA;
  }
  return BQCDG_OK;
}

// the reduction over all slabs of the partials the last second pass stored
// (nsb per slab, from slot 0 of each slab's RedScratch), applied by mode
// (1: alpha, 2: the CG step) to the shared scalars: in this process in slab
// order, then over the ranks by ncclAllReduce
int dd_reduce(bqcdg_dd* dd, int nsb, CgScalars* cg, int mode) {
  DdPartials parts{};
  for (int s = 0; s < dd->nslabs(); s++) parts.p[s] = dd->slabs[s]->red.partial;
  if (!dd->nccl) {
    launch_dd_total(parts, dd->nslabs(), nsb, cg, nullptr, mode, dd->stream);
    CKL();
    return BQCDG_OK;
  }
  launch_dd_total(parts, dd->nslabs(), nsb, cg, dd->dtot, 0, dd->stream);
  CKL();
  if (g_nccl.allReduce(dd->dtot, dd->dtot, 1, ncclDouble, ncclSum, dd->comm, dd->stream) != ncclSuccess)
    return BQCDG_ECUDA;
  launch_dd_apply(dd->dtot, cg, mode, dd->stream);
  CKL();
  return BQCDG_OK;
}

// U_t of each slab's last slice into the ghost links of the next slab
int dd_exchange_links(bqcdg_dd* dd) {
  const int n = dd->nslabs();
  if (!dd->nccl) {
    for (int s = 0; s < n; s++)
      launch_dd_pack_links(dd->slabs[s]->g, dd->geom(s), dd->slabs[s]->gauge64, dd->bufs[(s + 1) % n].ghost_link,
                           dd->stream);
    CKL();
    return BQCDG_OK;
  }
  SlabBufs& b = dd->bufs[0];
  launch_dd_pack_links(dd->slabs[0]->g, dd->geom(0), dd->slabs[0]->gauge64, b.send_links, dd->stream);
  CKL();
  const int r = dd->rank0, prev = (r + dd->nranks - 1) % dd->nranks, next = (r + 1) % dd->nranks;
  const size_t cnt = (size_t)18 * dd->V3h * 2;
  if (g_nccl.groupStart() != ncclSuccess) return BQCDG_ECUDA;
  ncclResult_t e = g_nccl.send(b.send_links, cnt, ncclDouble, next, dd->comm, dd->stream);
  if (e == ncclSuccess) e = g_nccl.recv(b.ghost_link, cnt, ncclDouble, prev, dd->comm, dd->stream);
  if (g_nccl.groupEnd() != ncclSuccess || e != ncclSuccess) return BQCDG_ECUDA;
  return BQCDG_OK;
}

// global sums of k local values per slab (dres[0..k-1] of each slab, written
// on dd->stream); out[0..k-1] on the host.  local: the slabs' values added in
// rank order; nccl: ncclAllReduce.
int dd_global_sum(bqcdg_dd* dd, int k, double* out) {
  if (!dd->nccl) {
    for (int j = 0; j < k; j++) out[j] = 0.0;
    CK(cudaStreamSynchronize(dd->stream));
    for (int s = 0; s < dd->nslabs(); s++) {
      double v[4];
      CK(cudaMemcpy(v, dd->slabs[s]->dres, k * sizeof(double), cudaMemcpyDeviceToHost));
      for (int j = 0; j < k; j++) out[j] += v[j];
    }
    return BQCDG_OK;
  }
  if (g_nccl.allReduce(dd->slabs[0]->dres, dd->dsum, k, ncclDouble, ncclSum, dd->comm, dd->stream) != ncclSuccess)
    return BQCDG_ECUDA;
  CK(cudaMemcpyAsync(out, dd->dsum, k * sizeof(double), cudaMemcpyDeviceToHost, dd->stream));
  CK(cudaStreamSynchronize(dd->stream));
  return BQCDG_OK;
}

double2* aee_of_slab(bqcdg_ctx* c) { return c->A[0]; }
double2* ainv_oo_of_slab(bqcdg_ctx* c) { return c->Ainv[1]; }

// out = mtil / mtil_dag in on every slab (t: odd work field of each slab)
int dd_mtil(bqcdg_dd* dd, bool dag, const std::vector<double2*>& out, const std::vector<double2*>& in,
            const std::vector<double2*>& t, const OpParams& op) {
  // the boundary slices on the exchange stream behind the faces, the
  // interior on the compute stream meanwhile, then the join
  int st;
  if ((st = dd_exchange(dd, in, dag))) return st;
  for (int part = 2; part >= 1; part--)
    for (int s = 0; s < dd->nslabs(); s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_dd_pass1(c->g, dd->geom(s), dag, t[s], in[s], c->gauge64, ainv_oo_of_slab(c), op,
                      part == 2 ? dd->xstream : dd->stream, part);
    }
  CKL();
  if ((st = dd_exchange_done(dd)) || (st = dd_wait_exchange(dd))) return st;
  if ((st = dd_exchange(dd, t, dag))) return st;
  for (int part = 2; part >= 1; part--)
    for (int s = 0; s < dd->nslabs(); s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_dd_pass2(c->g, dd->geom(s), dag, out[s], t[s], in[s], c->gauge64, aee_of_slab(c), op,
                      part == 2 ? dd->xstream : dd->stream, part);
    }
  CKL();
  if ((st = dd_exchange_done(dd)) || (st = dd_wait_exchange(dd))) return st;
  return BQCDG_OK;
}

int dd_mdagm(bqcdg_dd* dd, const std::vector<double2*>& out, const std::vector<double2*>& in,
             const std::vector<double2*>& t, const std::vector<double2*>& q, const OpParams& op) {
  int st = dd_mtil(dd, false, q, in, t, op);
  return st ? st : dd_mtil(dd, true, out, q, t, op);
}

// work field k of every slab
int dd_fields(bqcdg_dd* dd, int k, std::vector<double2*>& v) {
  v.resize(dd->nslabs());
  for (int s = 0; s < dd->nslabs(); s++)
    if (!(v[s] = dd->slabs[s]->sp64(k))) return BQCDG_ENOMEM;
  return BQCDG_OK;
}

// host spinors: local groups take the global array (slab s = rows
// [s volh_loc, (s+1) volh_loc)), nccl the slab's own
int dd_upload(bqcdg_dd* dd, const double* host, const std::vector<double2*>& dev) {
  for (int s = 0; s < dd->nslabs(); s++) {
    int st = upload_spinor(dd->slabs[s], host + (size_t)s * dd->volh_loc * 24, dev[s]);
    if (st) return st;
  }
  for (bqcdg_ctx* c : dd->slabs) CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}
int dd_download(bqcdg_dd* dd, const std::vector<double2*>& dev, double* host) {
  CK(cudaStreamSynchronize(dd->stream));
  for (int s = 0; s < dd->nslabs(); s++) {
    int st = download_spinor(dd->slabs[s], dev[s], host + (size_t)s * dd->volh_loc * 24);
    if (st) return st;
  }
  return BQCDG_OK;
}

int dd_create(bqcdg_dd** out, const int L[4], const int bc[4], int nranks, int rank, int nslabs, int device) {
  if (!out || !L || !bc || nranks < 1) return BQCDG_EINVAL;
  *out = nullptr;
  for (int d = 0; d < 4; d++)
    if (L[d] <= 0 || L[d] % 2 || (bc[d] != 1 && bc[d] != -1)) return BQCDG_EINVAL;
  if (L[3] % nranks || (L[3] / nranks) % 2) return BQCDG_EINVAL;  // even slabs keep the parity
  if (rank < 0 || rank + nslabs > nranks) return BQCDG_EINVAL;
  bqcdg_dd* dd = new bqcdg_dd();
  dd->nranks = nranks;
  dd->rank0 = rank;
  for (int d = 0; d < 4; d++) {
    dd->L[d] = L[d];
    dd->bc[d] = bc[d];
  }
  dd->Lt_loc = L[3] / nranks;
  dd->V3h = L[0] * L[1] * L[2] / 2;
  dd->volh_loc = dd->V3h * dd->Lt_loc;
  const int Lloc[4] = {L[0], L[1], L[2], dd->Lt_loc};
  for (int s = 0; s < nslabs; s++) {
    bqcdg_ctx* c = nullptr;
    int st = bqcdg_create(&c, Lloc, bc, device);
    if (st) {
      bqcdg_dd_destroy(dd);
      return st;
    }
    dd->slabs.push_back(c);
    dd->bufs.push_back(SlabBufs{});
  }
  dd->stream = dd->slabs[0]->stream;
  cudaError_t es = cudaSetDevice(device);
  if (es == cudaSuccess) es = cudaStreamCreateWithFlags(&dd->xstream, cudaStreamNonBlocking);
  if (es == cudaSuccess) es = cudaEventCreateWithFlags(&dd->ev_ready, cudaEventDisableTiming);
  if (es == cudaSuccess) es = cudaEventCreateWithFlags(&dd->ev_done, cudaEventDisableTiming);
  if (es != cudaSuccess) {
    bqcdg_dd_destroy(dd);
    return status_from_cuda(es);
  }
  const size_t face = (size_t)6 * dd->V3h * sizeof(double2), links = (size_t)18 * dd->V3h * sizeof(double2);
  for (int s = 0; s < nslabs; s++) {
    bqcdg_ctx* c = dd->slabs[s];
    SlabBufs& b = dd->bufs[s];
    cudaError_t e = c->alloc((void**)&b.ghost_fwd, face);
    if (e == cudaSuccess) e = c->alloc((void**)&b.ghost_bwd, face);
    if (e == cudaSuccess) e = c->alloc((void**)&b.ghost_link, links);
    if (e == cudaSuccess && s == 0) e = c->alloc((void**)&dd->dtot, 4 * sizeof(double));
    if (e != cudaSuccess) {
      bqcdg_dd_destroy(dd);
      return status_from_cuda(e);
    }
  }
  *out = dd;
  return BQCDG_OK;
}

}  // namespace

extern "C" {

int bqcdg_dd_create_local(bqcdg_dd** dd, const int L[4], const int bc[4], int nranks, int device) {
  return dd_create(dd, L, bc, nranks, 0, nranks, device);
}

int bqcdg_dd_nccl_unique_id(char* id) {
  if (!id) return BQCDG_EINVAL;
  if (!g_nccl.load()) return BQCDG_EUNSUPPORTED;
  ncclUniqueId u;
  if (g_nccl.getUniqueId(&u) != ncclSuccess) return BQCDG_ECUDA;
  std::memcpy(id, u.internal, sizeof(u.internal));
  return BQCDG_OK;
}

int bqcdg_dd_create_nccl(bqcdg_dd** out, const int L[4], const int bc[4], int nranks, int rank, int device,
                         const char* id) {
  if (!id) return BQCDG_EINVAL;
  if (!g_nccl.load()) return BQCDG_EUNSUPPORTED;
  int st = dd_create(out, L, bc, nranks, rank, 1, device);
  if (st) return st;
  bqcdg_dd* dd = *out;
  dd->nccl = true;
  bqcdg_ctx* c = dd->slabs[0];
  SlabBufs& b = dd->bufs[0];
  const size_t face = (size_t)6 * dd->V3h * sizeof(double2), links = (size_t)18 * dd->V3h * sizeof(double2);
  cudaError_t e = c->alloc((void**)&b.send_prev, face);
  if (e == cudaSuccess) e = c->alloc((void**)&b.send_next, face);
  if (e == cudaSuccess) e = c->alloc((void**)&b.send_links, links);
  if (e == cudaSuccess) e = c->alloc((void**)&dd->dsum, 4 * sizeof(double));
  ncclUniqueId u;
  std::memcpy(u.internal, id, sizeof(u.internal));
  if (e == cudaSuccess && g_nccl.commInitRank(&dd->comm, nranks, u, rank) != ncclSuccess) e = cudaErrorUnknown;
  if (e != cudaSuccess) {
    bqcdg_dd_destroy(dd);
    *out = nullptr;
    return BQCDG_ECUDA;
  }
  return BQCDG_OK;
}

int bqcdg_dd_destroy(bqcdg_dd* dd) {
  if (!dd) return BQCDG_EINVAL;
  if (dd->comm) g_nccl.commDestroy(dd->comm);
  if (dd->xstream) cudaStreamSynchronize(dd->xstream);
  if (dd->ev_ready) cudaEventDestroy(dd->ev_ready);
  if (dd->ev_done) cudaEventDestroy(dd->ev_done);
  if (dd->xstream) cudaStreamDestroy(dd->xstream);
  for (bqcdg_ctx* c : dd->slabs) bqcdg_destroy(c);  // frees every buffer the slab allocated
  delete dd;
  return BQCDG_OK;
}

int bqcdg_dd_volh(const bqcdg_dd* dd) { return dd ? dd->volh_loc * (int)dd->slabs.size() : -1; }

int bqcdg_dd_load_gauge(bqcdg_dd* dd, const double* u, int flipped) {
  int st = dd_check(dd);
  if (st || !u) return BQCDG_EINVAL;
  const size_t nloc = (size_t)dd->volh_loc * 18;  // doubles of one (mu, parity) block of a slab
  const size_t nhost = nloc * dd->nslabs();
  std::vector<double> tmp(8 * nloc);
  for (int s = 0; s < dd->nslabs(); s++) {
    for (int me = 0; me < 8; me++) std::memcpy(tmp.data() + me * nloc, u + me * nhost + s * nloc, nloc * 8);
    // only the last slab holds the global last time slice, where flip_bc put its sign
    const bool last = dd->rank0 + s == dd->nranks - 1;
    if ((st = bqcdg_load_gauge(dd->slabs[s], tmp.data(), flipped && last ? 1 : 0))) return st;
  }
  if ((st = dd_exchange_links(dd))) return st;
  CK(cudaStreamSynchronize(dd->stream));
  return BQCDG_OK;
}

int bqcdg_dd_load_clover(bqcdg_dd* dd, const double* a, const double* ainv) {
  int st = dd_check(dd);
  if (st || !a || !ainv) return BQCDG_EINVAL;
  const size_t nloc = (size_t)dd->volh_loc * 72;  // doubles of one parity of a slab
  const size_t nhost = nloc * dd->nslabs();
  std::vector<double> ta(2 * nloc), ti(2 * nloc);
  for (int s = 0; s < dd->nslabs(); s++) {
    for (int eo = 0; eo < 2; eo++) {
      std::memcpy(ta.data() + eo * nloc, a + eo * nhost + s * nloc, nloc * 8);
      std::memcpy(ti.data() + eo * nloc, ainv + eo * nhost + s * nloc, nloc * 8);
    }
    if ((st = bqcdg_load_clover(dd->slabs[s], ta.data(), ti.data(), nullptr))) return st;
    CK(cudaStreamSynchronize(dd->slabs[s]->stream));
  }
  return BQCDG_OK;
}

int bqcdg_dd_op(bqcdg_dd* dd, int which, double* out, const double* in, const bqcdg_params* p) {
  int st = dd_check(dd);
  if (st || !out || !in || !p || which < 0 || which > 7) return BQCDG_EINVAL;
  for (bqcdg_ctx* c : dd->slabs) {
    if (!c->have_gauge) return BQCDG_ENOGAUGE;
    if (p->csw_kappa != 0.0 && which < 6 && (!c->have_A[0] || !c->have_Ainv[1])) return BQCDG_ENOCLOVER;
  }
  CK(cudaSetDevice(dd->slabs[0]->device));
  std::vector<double2*> vin, vout, t, q;
  if ((st = dd_fields(dd, 0, vin)) || (st = dd_fields(dd, 1, vout)) || (st = dd_fields(dd, 2, t)) ||
      (st = dd_fields(dd, 3, q)))
    return st;
  if ((st = dd_upload(dd, in, vin))) return st;
  const bool w = which >= 3 && which <= 5;
  OpParams op = op_of(p, w);
  switch (which) {
    case 0: case 3: st = dd_mtil(dd, false, vout, vin, t, op); break;
    case 1: case 4: st = dd_mtil(dd, true, vout, vin, t, op); break;
    case 2: case 5: st = dd_mdagm(dd, vout, vin, t, q, op); break;
    default:  // 6: d(EVEN, ODD), 7: d_dag(EVEN, ODD)
      if ((st = dd_exchange(dd, vin, which == 7)) || (st = dd_exchange_done(dd)) || (st = dd_wait_exchange(dd)))
        break;
      for (int s = 0; s < dd->nslabs(); s++)
        launch_dd_dslash(dd->slabs[s]->g, dd->geom(s), 0, which == 7, vout[s], vin[s], dd->slabs[s]->gauge64,
                         dd->stream);
      st = cudaGetLastError() == cudaSuccess ? BQCDG_OK : BQCDG_ECUDA;
  }
  if (st) return st;
  return dd_download(dd, vout, out);
}

// cg.F90:51-137 over the slabs: FP64, x the initial guess, absolute stop
// rtr <= cgp->rest, (W^+W) with W = M~ + p->rho; the three scalars of each
// iteration are global sums (cg.F90:91,97,109)
int bqcdg_dd_cg(bqcdg_dd* dd, double* x, const double* b, const bqcdg_params* p, const bqcdg_cg_para* cgp,
                int* iterations, bqcdg_solve_info* info) {
  int st = dd_check(dd);
  if (st || !x || !b || !p || !cgp) return BQCDG_EINVAL;
  for (bqcdg_ctx* c : dd->slabs) {
    if (!c->have_gauge) return BQCDG_ENOGAUGE;
    if (p->csw_kappa != 0.0 && (!c->have_A[0] || !c->have_Ainv[1])) return BQCDG_ENOCLOVER;
  }
  CK(cudaSetDevice(dd->slabs[0]->device));
  bqcdg_solve_info tmp;
  if (!info) info = &tmp;
  std::memset(info, 0, sizeof(*info));
  std::vector<double2*> vx, vb, vr, vp, vap, t, q;
  if ((st = dd_fields(dd, 0, vx)) || (st = dd_fields(dd, 1, vb)) || (st = dd_fields(dd, 2, vr)) ||
      (st = dd_fields(dd, 3, vp)) || (st = dd_fields(dd, 4, vap)) || (st = dd_fields(dd, 5, t)) ||
      (st = dd_fields(dd, 6, q)))
    return st;
  if ((st = dd_upload(dd, x, vx)) || (st = dd_upload(dd, b, vb))) return st;
  const OpParams op = op_of(p, true);
  const int n = dd->nslabs();
  EventPair ev;
  CK(ev.create());
  cudaEvent_t e0 = ev.e0, e1 = ev.e1;
  CK(cudaEventRecord(e0, dd->stream));
  auto dot = [&](const std::vector<double2*>& a, const std::vector<double2*>& c2, double* out) {
    for (int s = 0; s < n; s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_dot(c->g, a[s], c2[s], c->red, c->dres, dd->stream);
    }
    if (cudaGetLastError() != cudaSuccess) return BQCDG_ECUDA;
    return dd_global_sum(dd, 1, out);
  };
  // r = b - A x, p = r
  if ((st = dd_mdagm(dd, vr, vx, t, q, op))) return st;
  for (int s = 0; s < n; s++) {
    bqcdg_ctx* c = dd->slabs[s];
    launch_caxpby(c->g, 1.0, 0.0, vb[s], -1.0, vr[s], dd->stream);  // r = b - r
    CK(cudaMemcpyAsync(vp[s], vr[s], (size_t)12 * c->g.stride * sizeof(double2), cudaMemcpyDeviceToDevice,
                       dd->stream));
  }
  CKL();
  double rtrold = 0.0, rtr = 0.0, paap = 0.0;
  if ((st = dot(vr, vr, &rtrold))) return st;
  int niter = 0;
  bool conv = false;
  for (niter = 1; niter <= cgp->maxiter; niter++) {
    if ((st = dd_mdagm(dd, vap, vp, t, q, op))) return st;
    if ((st = dot(vp, vap, &paap))) return st;
    const double ak = rtrold / paap;
    for (int s = 0; s < n; s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_axpy(c->g, ak, vp[s], vx[s], dd->stream);
      launch_axpy(c->g, -ak, vap[s], vr[s], dd->stream);
    }
    CKL();
    if ((st = dot(vr, vr, &rtr))) return st;
    if (!(rtr == rtr)) break;
    if (rtr <= (double)cgp->rest) {
      conv = true;
      break;
    }
    const double bk = rtr / rtrold;
    rtrold = rtr;
    for (int s = 0; s < n; s++) launch_caxpby(dd->slabs[s]->g, 1.0, 0.0, vr[s], bk, vp[s], dd->stream);  // p = r + bk p
    CKL();
  }
  if (!conv && niter > cgp->maxiter) niter = cgp->maxiter;
  CK(cudaEventRecord(e1, dd->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if ((st = dd_download(dd, vx, x))) return st;
  info->niter = niter;
  info->rtr = rtr;
  info->converged = conv ? 1 : 0;
  info->seconds = ms * 1e-3;
  if (iterations) *iterations = niter;
  if (!(rtr == rtr)) return BQCDG_ENAN;
  if (!conv && cgp->log != 2) return BQCDG_ENOCONV;
  return BQCDG_OK;
}

// The mixed-precision solve over the slabs: the scheme of cg_core (capi.cu)
// -- int16 sloppy iterations, FP32 r and x_s, FP64 reliable updates when |r|
// has fallen by o->delta, p re-orthogonalised after each -- with every
// stencil pass split around the face exchange (the boundary slices behind
// the faces on the exchange stream, the interior on the compute stream) and
// the two reductions of an iteration summed over all slabs (dd_reduce) into
// one set of CG scalars on the device, so the iterations never wait for the
// host.
int bqcdg_dd_solve(bqcdg_dd* dd, double* x, const double* b, const bqcdg_params* p, const bqcdg_solver_opts* o,
                   bqcdg_solve_info* info) {
  int st = dd_check(dd);
  if (st || !x || !b || !p || !o || !info) return BQCDG_EINVAL;
  if (o->precision != BQCDG_PREC_HALF) return BQCDG_EUNSUPPORTED;  // FP64: bqcdg_dd_cg
  if (dd->nslabs() > kMaxDdSlabs || o->delta <= 0.0 || o->delta >= 1.0) return BQCDG_EINVAL;
  const bool clover = p->csw_kappa != 0.0;
  for (bqcdg_ctx* c : dd->slabs) {
    if (!c->have_gauge) return BQCDG_ENOGAUGE;
    if (clover && (!c->have_A[0] || !c->have_Ainv[1])) return BQCDG_ENOCLOVER;
  }
  CK(cudaSetDevice(dd->slabs[0]->device));
  std::memset(info, 0, sizeof(*info));
  const int n = dd->nslabs();
  const Prec P = Prec::F16;
  for (bqcdg_ctx* c : dd->slabs)
    if ((st = ensure_sloppy(c, P, clover))) return st;
  std::vector<double2*> vx, vb, vr, vax, t64, q64;
  if ((st = dd_fields(dd, 0, vx)) || (st = dd_fields(dd, 1, vb)) || (st = dd_fields(dd, 2, vr)) ||
      (st = dd_fields(dd, 3, vax)) || (st = dd_fields(dd, 4, t64)) || (st = dd_fields(dd, 5, q64)))
    return st;
  std::vector<SpinorPtr> sp(n), tf(n), sq(n), rs(n), xs(n);
  for (int s = 0; s < n; s++) {
    bqcdg_ctx* c = dd->slabs[s];
    sp[s] = c->sp(P, 0);
    tf[s] = c->sp(P, 1);
    sq[s] = c->sp(P, 2);
    rs[s] = c->sp(Prec::F32, 0);
    xs[s] = c->sp(Prec::F32, 1);
    if (!sp[s].v || !tf[s].v || !sq[s].v || !rs[s].v || !xs[s].v) return BQCDG_ENOMEM;
  }
  if ((st = dd_upload(dd, x, vx)) || (st = dd_upload(dd, b, vb))) return st;
  const OpParams op = op_of(p, true);
  bqcdg_ctx* c0 = dd->slabs[0];
  CgScalars* dcg = c0->dcg;  // the scalars every slab's kernels read
  EventPair ev;
  CK(ev.create());
  cudaEvent_t e0 = ev.e0, e1 = ev.e1;
  CK(cudaEventRecord(e0, dd->stream));

  // r = b - A x in FP64 and |r|^2, |b|^2 over the slabs
  auto residual = [&](double* r2b2) -> int {
    int s2 = dd_mdagm(dd, vax, vx, t64, q64, op);
    if (s2) return s2;
    for (int s = 0; s < n; s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_residual(c->g, vr[s], vb[s], vax[s], Prec::F32, rs[s], c->red, c->dres, dd->stream);
    }
    CKL();
    return dd_global_sum(dd, 2, r2b2);
  };
  double rb[2];
  if ((st = residual(rb))) return st;
  const double b2 = rb[1];
  const double stop = o->relative ? o->tol * o->tol * b2 : o->tol;
  info->b2 = b2;
  for (int s = 0; s < n; s++) {
    launch_spinor_convert(dd->slabs[s]->g, P, sp[s], Prec::F32, rs[s], dd->stream);
    launch_zero(dd->slabs[s]->g, Prec::F32, xs[s], dd->stream);
  }
  CKL();
  CgScalars h{};
  h.rtr = h.rtr_old = rb[0];
  h.stop_rtr = stop;
  h.maxiter = o->maxiter;
  h.delta2 = o->delta * o->delta;
  h.maxr2 = rb[0];
  h.ru_every = 500;  // periodic reliable updates of the int16 iterations, as in cg_core
  bool converged = false;
  if (!(rb[0] == rb[0])) h.done = 4;
  else if (rb[0] == 0.0 || rb[0] <= stop) { h.done = 1; converged = true; }
  if (o->maxiter <= 0 && !h.done) h.done = 3;
  auto put = [&]() -> int {
    CK(cudaMemcpyAsync(dcg, &h, sizeof(h), cudaMemcpyHostToDevice, dd->stream));
    CK(cudaStreamSynchronize(dd->stream));
    return BQCDG_OK;
  };
  auto get = [&]() -> int {
    CK(cudaMemcpyAsync(&h, dcg, sizeof(h), cudaMemcpyDeviceToHost, dd->stream));
    CK(cudaStreamSynchronize(dd->stream));
    return BQCDG_OK;
  };
  if ((st = put())) return st;
  // one stencil pass: the faces of xf exchanged on xstream and the boundary
  // slices queued behind them there, the interior slices on the compute
  // stream meanwhile, then the join
  auto pass = [&](const std::vector<SpinorPtr>& xf, bool dag, auto launch_part) -> int {
    int s2 = dd_exchange16(dd, xf, dag);
    if (s2) return s2;
    for (int part = 2; part >= 1; part--)
      for (int s = 0; s < n; s++) launch_part(s, part, part == 2 ? dd->xstream : dd->stream);
    CKL();
    if ((s2 = dd_exchange_done(dd)) || (s2 = dd_wait_exchange(dd))) return s2;
    return BQCDG_OK;
  };
  const int nsb1 = nblocks(dd_part_sites(1, dd->Lt_loc, dd->V3h));
  const int nparts = nsb1 > 0 ? 2 : 1;  // a slab of two slices has no interior launch
  const int nsb = nsb1 + nblocks(dd_part_sites(2, dd->Lt_loc, dd->V3h));
  int batch = 4, ru = 0, stall = 0, forced = 0, launches = 0;
  double best = rb[0];
  bool stalled = false;
  while (!h.done) {
    const int iter0 = h.iter;
    for (int k = 0; k < batch; k++) {
      // pass 1: t = A_oo^-1 D_oe p
      st = pass(sp, false, [&](int s, int part, cudaStream_t str) {
        bqcdg_ctx* c = dd->slabs[s];
        launch_dd16_pass1(c->g, dd->geom(s), false, part, tf[s], sp[s], gauge_of(c, P), ainv_of(c, P), op, dcg,
                          str);
      });
      if (st) return st;
      // pass 2: q = M~ p, |q|^2 -> alpha
      st = pass(tf, false, [&](int s, int part, cudaStream_t str) {
        bqcdg_ctx* c = dd->slabs[s];
        launch_dd16_pass2(c->g, dd->geom(s), false, part, sq[s], tf[s], sp[s], gauge_of(c, P), aee_of(c, P), op,
                          c->red.partial, part == 1 ? 0 : nsb1, dcg, str);
      });
      if (st || (st = dd_reduce(dd, nsb, dcg, 1))) return st;
      // pass 3: t = A_oo^-1 D^+_oe q
      st = pass(sq, true, [&](int s, int part, cudaStream_t str) {
        bqcdg_ctx* c = dd->slabs[s];
        launch_dd16_pass1(c->g, dd->geom(s), true, part, tf[s], sq[s], gauge_of(c, P), ainv_of(c, P), op, dcg,
                          str);
      });
      if (st) return st;
      // pass 4: A p, r -= alpha A p, |r|^2 -> the CG step
      st = pass(tf, true, [&](int s, int part, cudaStream_t str) {
        bqcdg_ctx* c = dd->slabs[s];
        launch_dd16_pass4(c->g, dd->geom(s), part, tf[s], sq[s], gauge_of(c, P), aee_of(c, P), op, rs[s],
                          c->red.partial, part == 1 ? 0 : nsb1, dcg, str);
      });
      if (st || (st = dd_reduce(dd, nsb, dcg, 2))) return st;
      // x += alpha p of this iteration if it ran, p = r + beta p if the solve goes on
      for (int s = 0; s < n; s++)
        launch_cg_pupdate(P, dd->slabs[s]->g, sp[s], rs[s], dcg, dd->stream, 1, xs[s], iter0 + k + 1);
      CKL();
      launches += 4 * (n + nparts * n) + 2 * (dd->nccl ? 2 : 1) + n;
    }
    if ((st = get())) return st;
    if (batch < 16) batch *= 2;
    if (h.done == 4) break;
    if (h.done == 0) continue;
    // reliable update: x += x_s, r = b - A x in FP64 over the slabs
    const bool periodic = !(h.rtr < h.delta2 * h.maxr2);
    for (int s = 0; s < n; s++) launch_accum_x(dd->slabs[s]->g, vx[s], (float4*)xs[s].v, dd->stream);
    CKL();
    if ((st = residual(rb))) return st;
    ru++;
    const double rtrue = rb[0];
    if (!(rtrue == rtrue)) { h.done = 4; break; }
    if (rtrue <= stop) { h.rtr = rtrue; converged = true; h.done = 1; break; }
    if (h.done == 3) { h.rtr = rtrue; break; }
    if (rtrue < 0.5 * best) { best = rtrue; stall = 0; }
    else if (++stall >= 5 || rtrue > 1e4 * best) { h.rtr = rtrue; stalled = true; break; }
    forced = periodic ? forced + 1 : 0;
    if (forced >= 2) { h.rtr = rtrue; stalled = true; break; }
    // continue from the true residual with p re-orthogonalised against it
    for (int s = 0; s < n; s++) {
      bqcdg_ctx* c = dd->slabs[s];
      launch_rdot(c->g, rs[s], P, sp[s], c->red, c->dres, dd->stream);
    }
    CKL();
    double rp;
    if ((st = dd_global_sum(dd, 1, &rp))) return st;
    const double rpc = rp / rtrue;
    h.beta = rtrue / h.rtr_old;
    h.rtr = rtrue;
    h.maxr2 = rtrue;
    h.last_ru = h.iter;
    h.done = 0;
    if ((st = put())) return st;
    for (int s = 0; s < n; s++) launch_p_reorth(dd->slabs[s]->g, P, sp[s], rs[s], rpc, h.beta, dd->stream);
    CKL();
  }
  CK(cudaEventRecord(e1, dd->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if ((st = dd_download(dd, vx, x))) return st;
  info->seconds = ms * 1e-3;
  info->niter = h.iter;
  info->reliable_updates = ru;
  info->kernel_launches = launches;
  info->rtr = h.rtr;
  info->true_rtr = h.rtr;
  info->converged = converged ? 1 : 0;
  if (h.done == 4) return BQCDG_ENAN;
  if (stalled || !converged) return BQCDG_ENOCONV;
  return BQCDG_OK;
}

}  // extern "C"
