// Halo exchange of a z-slab decomposition over NCCL: the analogue of the
// driver's SYNC (AsterX/schedule.ccl:110-115,157-164) between the ranks that
// each hold one z-slab of a periodic patch, one process per GPU.
//
// A k-plane of the engine's layout is contiguous (f[i + sy j + sz k]), so the
// halo of a field is two runs of ng planes.  One exchange packs the planes of
// every listed field into one buffer per direction (one kernel), sends and
// receives them as one NCCL group of four point-to-point operations over
// NVLink, and unpacks them into the ghost planes (one kernel).  Plane
// mapping, with nz this rank's interior cells and v = 1 for a field that is
// vertex-centred in z: the lower ghosts [0, ng) take the lower neighbour's
// planes [nz, nz + ng) (sent "up"), the upper ghosts [ng + nz + v,
// 2 ng + nz + v) take the upper neighbour's planes [ng + v, 2 ng + v) (sent
// "down").  With one rank the exchange is the periodic wrap in z.
#include <cstring>
#include <mutex>
#include <new>

#include <dlfcn.h>
#include <nccl.h>

#include "axb_internal.hxx"

// NCCL is resolved at run time, not linked: a process that has imported a
// framework carries its own libnccl, and a second copy bound at load time
// would shadow the symbols that framework expects.  The entry points take
// the NCCL the process has loaded, else libnccl.so.2.
namespace {
struct Nccl {
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t,
                       cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t,
                       cudaStream_t) = nullptr;
  bool ok = false;
};
const Nccl &nccl() {
  static Nccl n;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = RTLD_DEFAULT;
    if (!dlsym(h, "ncclGetUniqueId"))
      h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h)
      return;
    n.GetUniqueId = reinterpret_cast<decltype(n.GetUniqueId)>(dlsym(h, "ncclGetUniqueId"));
    n.CommInitRank = reinterpret_cast<decltype(n.CommInitRank)>(dlsym(h, "ncclCommInitRank"));
    n.CommDestroy = reinterpret_cast<decltype(n.CommDestroy)>(dlsym(h, "ncclCommDestroy"));
    n.GroupStart = reinterpret_cast<decltype(n.GroupStart)>(dlsym(h, "ncclGroupStart"));
    n.GroupEnd = reinterpret_cast<decltype(n.GroupEnd)>(dlsym(h, "ncclGroupEnd"));
    n.Send = reinterpret_cast<decltype(n.Send)>(dlsym(h, "ncclSend"));
    n.Recv = reinterpret_cast<decltype(n.Recv)>(dlsym(h, "ncclRecv"));
    n.ok = n.GetUniqueId && n.CommInitRank && n.CommDestroy && n.GroupStart && n.GroupEnd &&
           n.Send && n.Recv;
  });
  return n;
}
} // namespace

namespace axb {
int gf_centring(int gf, int c[3]);
} // namespace axb

struct axb_halo {
  int device = 0, rank = 0, nranks = 1, up = 0, down = 0;
  ncclComm_t comm = nullptr;
  axb_box box{};
  int nf = 0;
  int ids[AXB_NUM_GF];
  int vz[AXB_NUM_GF]; // 1: vertex-centred in z
  size_t seg = 0;     // ng planes, elements
  double *buf = nullptr; // send up, send down, receive low, receive high
};

namespace {

struct HaloCopies {
  double *f[AXB_NUM_GF];
  int vz[AXB_NUM_GF];
  int nf;
  long long seg, plane, nz, ng;
  double *send_up, *send_down, *recv_low, *recv_high;
};

// one thread per element of the nf x seg planes of each direction
__global__ void __launch_bounds__(256) k_halo_pack(const HaloCopies h) {
  const long long n = (long long)h.nf * h.seg;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = int(e / h.seg);
    const long long o = e - (long long)q * h.seg;
    const double *f = h.f[q];
    h.send_up[e] = f[h.nz * h.plane + o];
    h.send_down[e] = f[(h.ng + h.vz[q]) * h.plane + o];
  }
}

__global__ void __launch_bounds__(256) k_halo_unpack(const HaloCopies h) {
  const long long n = (long long)h.nf * h.seg;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = int(e / h.seg);
    const long long o = e - (long long)q * h.seg;
    double *f = h.f[q];
    f[o] = h.recv_low[e];
    f[(h.ng + h.nz + h.vz[q]) * h.plane + o] = h.recv_high[e];
  }
}

} // namespace

// ncclGetUniqueId: rank 0 makes the id, the caller's launcher hands it to
// every rank (e.g. torch.distributed.broadcast_object_list).
AXB_API int axb_halo_unique_id(unsigned char id[128]) {
  static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id size");
  if (!id)
    return AXB_ERR_ARG;
  const Nccl &N = nccl();
  if (!N.ok)
    return AXB_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (N.GetUniqueId(&u) != ncclSuccess)
    return AXB_ERR_CUDA;
  std::memcpy(id, &u, sizeof u);
  return AXB_OK;
}

AXB_API int axb_halo_create(axb_ctx *c, const axb_box *box, int nranks, int rank,
                            const unsigned char id[128], const int *field_ids, int nfields,
                            axb_halo **out) {
  if (!c || !box || !id || !field_ids || !out || nranks < 1 || rank < 0 || rank >= nranks ||
      nfields < 1 || nfields > AXB_NUM_GF)
    return AXB_ERR_ARG;
  *out = nullptr;
  if (box->ng < 1 || box->n[2] < box->ng || box->sz < 1)
    return AXB_ERR_ARG;
  const Nccl &N = nccl();
  if (!N.ok)
    return AXB_ERR_UNSUPPORTED;
  axb_halo *h = new (std::nothrow) axb_halo();
  if (!h)
    return AXB_ERR_ARG;
  h->device = c->device;
  h->rank = rank;
  h->nranks = nranks;
  h->up = (rank + 1) % nranks;
  h->down = (rank + nranks - 1) % nranks;
  h->box = *box;
  h->nf = nfields;
  for (int q = 0; q < nfields; ++q) {
    if (field_ids[q] < 0 || field_ids[q] >= AXB_NUM_GF) {
      delete h;
      return AXB_ERR_ARG;
    }
    int cent[3];
    axb::gf_centring(field_ids[q], cent);
    h->ids[q] = field_ids[q];
    h->vz[q] = cent[2] ? 0 : 1;
  }
  h->seg = size_t(box->ng) * size_t(box->sz);
  if (cudaSetDevice(c->device) != cudaSuccess ||
      cudaMalloc(&h->buf, 4 * size_t(nfields) * h->seg * sizeof(double)) != cudaSuccess) {
    delete h;
    return AXB_ERR_CUDA;
  }
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof u);
  if (N.CommInitRank(&h->comm, nranks, u, rank) != ncclSuccess) {
    cudaFree(h->buf);
    delete h;
    return AXB_ERR_CUDA;
  }
  *out = h;
  return AXB_OK;
}

AXB_API int axb_halo_exchange(axb_halo *h, const axb_fields *f, void *stream) {
  if (!h || !f)
    return AXB_ERR_ARG;
  HaloCopies k{};
  for (int q = 0; q < h->nf; ++q) {
    k.f[q] = f->gf[h->ids[q]];
    k.vz[q] = h->vz[q];
    if (!k.f[q])
      return AXB_ERR_ARG;
  }
  k.nf = h->nf;
  k.seg = (long long)h->seg;
  k.plane = h->box.sz;
  k.nz = h->box.n[2];
  k.ng = h->box.ng;
  const size_t n = size_t(h->nf) * h->seg;
  k.send_up = h->buf;
  k.send_down = h->buf + n;
  k.recv_low = h->buf + 2 * n;
  k.recv_high = h->buf + 3 * n;
  cudaStream_t s = (cudaStream_t)stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  const long long want = ((long long)n + 255) / 256;
  const unsigned blocks = unsigned(want < 8LL * sms ? want : 8LL * sms);
  k_halo_pack<<<blocks, 256, 0, s>>>(k);
  if (cudaGetLastError() != cudaSuccess)
    return AXB_ERR_CUDA;
  // the upper planes go up and arrive as the upper neighbour's lower ghosts;
  // the lower planes go down
  const Nccl &N = nccl();
  if (N.GroupStart() != ncclSuccess)
    return AXB_ERR_CUDA;
  // a group once opened is always closed, whatever failed inside it
  const bool queued =
      N.Send(k.send_up, n, ncclDouble, h->up, h->comm, s) == ncclSuccess &&
      N.Recv(k.recv_low, n, ncclDouble, h->down, h->comm, s) == ncclSuccess &&
      N.Send(k.send_down, n, ncclDouble, h->down, h->comm, s) == ncclSuccess &&
      N.Recv(k.recv_high, n, ncclDouble, h->up, h->comm, s) == ncclSuccess;
  if (N.GroupEnd() != ncclSuccess || !queued)
    return AXB_ERR_CUDA;
  k_halo_unpack<<<blocks, 256, 0, s>>>(k);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

AXB_API int axb_halo_destroy(axb_halo *h) {
  if (!h)
    return AXB_ERR_ARG;
  if (h->comm)
    nccl().CommDestroy(h->comm);
  cudaFree(h->buf);
  delete h;
  return AXB_OK;
}
