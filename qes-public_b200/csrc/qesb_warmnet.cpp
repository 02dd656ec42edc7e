// The learned warm start behind the C ABI: loads a trained network
// (qesb_warmnet_load), predicts lambda for a handle's inputs and sets it as
// the handle's starting lambda (qesb_warm_start). The layer loop, buffers and
// weight layouts live here; every convolution, pooling, input and apply step
// is one of the library's kernels, called through its C entry points, on the
// handle's stream.
//
// Network (the one qes-public_b200/qesb/warmstart.py trains): levels
// l = 0..L-1 with channels C[l] on the net grid divided by 2^l. Encoder: two
// 3x3x3 convolutions (ReLU) per level, 2x2x2 average pooling between levels.
// Decoder, l = L-2 .. 0: a convolution of [nearest-upsampled level l+1,
// skip e_l], then a second convolution. Head: one convolution to 16 FP32
// channels, channel 0 being lambda / max|R|. With res = 2 the net grid is the
// cell grid halved in every direction (features pooled, prediction applied by
// trilinear interpolation).
//
// Weights file (little-endian): "QESBWNT1", int32 nlev, res, in_ch, head_n,
// int32 channels[nlev], then per layer in the order e0a, e0, ..., e{L-1}a,
// e{L-1}, d{L-2}a, d{L-2}, ..., d0a, d0, head: int32 c1, c2, cout, cout_real,
// relu, up1, float W[27 (c1 + c2) cout] (row tap (c1 + c2) + c, column
// output channel), float b[cout].
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "qesb.h"
#include "qesb_internal.h"

namespace {

constexpr int kInCh = 16;   // network input channels (5 used)
constexpr int kHeadN = 16;  // head width (channel 0 is the prediction)

struct Layer {
  int c1 = 0, c2 = 0, cout = 0, cout_real = 0, relu = 0, up1 = 0, Kp = 0;
  uint16_t *Bm = nullptr;  // BF16 [cout][Kp], device
  float *bias = nullptr;   // [cout], device
};

// Activations of one net grid shape (D, H, W at level 0), BF16 channels-last.
struct Buffers {
  uint16_t *x = nullptr;
  float *y = nullptr;
  std::vector<uint16_t *> ea, e, p, da, d;
};

uint16_t bf16_rn(float f)
{
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
  u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest, ties to even
  return (uint16_t)(u >> 16);
}

}  // namespace

struct qesb_warmnet {
  int device = 0, nlev = 0, res = 1;
  std::vector<int> ch;
  std::vector<Layer> layers;  // file order
  int *d_err = nullptr;
  int *h_err = nullptr, *h_err_dev = nullptr;  // mapped pinned copy of *d_err, and its device alias
  unsigned *d_scale = nullptr;    // [nscale] max|R| per item of a call
  int nscale = 0;
  cudaEvent_t ev = nullptr;       // orders a batch's per-handle streams with the forward's stream
  std::map<std::tuple<int, int, int>, Buffers> bufs;
  std::vector<void *> owned;
  std::mutex mu;

  qesb_status alloc(void **p, size_t bytes)
  {
    if (cudaMalloc(p, bytes) != cudaSuccess) return qesb_fail(QESB_ERR_NOMEM, "qesb_warmnet: cudaMalloc of %zu bytes", bytes);
    owned.push_back(*p);
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_warmnet: cudaMemset");
    return QESB_OK;
  }

  int index(char kind, int l, bool a) const
  {
    // e0a, e0, e1a, e1, ... then d{L-2}a, d{L-2}, ..., d0a, d0, then head
    if (kind == 'e') return 2 * l + (a ? 0 : 1);
    if (kind == 'd') return 2 * nlev + 2 * (nlev - 2 - l) + (a ? 0 : 1);
    return 2 * nlev + 2 * (nlev - 1);
  }

  qesb_status buffers(int D, int H, int W, Buffers **out)
  {
    auto key = std::make_tuple(D, H, W);
    auto it = bufs.find(key);
    if (it != bufs.end()) {
      *out = &it->second;
      return QESB_OK;
    }
    Buffers b;
    auto V = [&](int l) { return (size_t)(D >> l) * (size_t)(H >> l) * (size_t)(W >> l); };
    void *p = nullptr;
    CKS_FWD(alloc(&p, V(0) * kInCh * 2));
    b.x = static_cast<uint16_t *>(p);
    CKS_FWD(alloc(&p, V(0) * 4));  // the head's prediction channel
    b.y = static_cast<float *>(p);
    b.ea.resize(nlev);
    b.e.resize(nlev);
    b.p.assign(nlev, nullptr);
    b.da.assign(nlev, nullptr);
    b.d.assign(nlev, nullptr);
    for (int l = 0; l < nlev; ++l) {
      CKS_FWD(alloc(&p, V(l) * ch[l] * 2));
      b.ea[l] = static_cast<uint16_t *>(p);
      CKS_FWD(alloc(&p, V(l) * ch[l] * 2));
      b.e[l] = static_cast<uint16_t *>(p);
      if (l > 0) {
        CKS_FWD(alloc(&p, V(l) * ch[l - 1] * 2));
        b.p[l] = static_cast<uint16_t *>(p);
      }
      if (l < nlev - 1) {
        CKS_FWD(alloc(&p, V(l) * ch[l] * 2));
        b.da[l] = static_cast<uint16_t *>(p);
        CKS_FWD(alloc(&p, V(l) * ch[l] * 2));
        b.d[l] = static_cast<uint16_t *>(p);
      }
    }
    *out = &bufs.emplace(key, b).first->second;
    return QESB_OK;
  }

  qesb_status conv(const Layer &L, const void *x1, const void *x2, int items, int D, int H, int W, void *y,
                   void *yf, void *stream)
  {
    return qesb_conv3d_items(x1, L.c1, L.up1, x2, L.c2, items, D, H, W, 1, L.Bm, L.Kp, L.cout, y, yf, L.bias,
                             L.relu, nullptr, d_err, stream);
  }

  // forward pass on b.x (`items` net grids of D x H x W stacked along z) into b.y
  qesb_status forward(Buffers &b, int items, int D, int H, int W, void *s)
  {
    for (int l = 0; l < nlev; ++l) {
      const int Dl = D >> l, Hl = H >> l, Wl = W >> l;
      const void *xin = b.x;
      if (l > 0) {  // the items' depths are even: no 2x2x2 block spans two of them
        CKS_FWD(qesb_net_pool2(b.e[l - 1], b.p[l], items * (D >> (l - 1)), H >> (l - 1), W >> (l - 1), ch[l - 1], s));
        xin = b.p[l];
      }
      CKS_FWD(conv(layers[index('e', l, true)], xin, nullptr, items, Dl, Hl, Wl, b.ea[l], nullptr, s));
      CKS_FWD(conv(layers[index('e', l, false)], b.ea[l], nullptr, items, Dl, Hl, Wl, b.e[l], nullptr, s));
    }
    for (int l = nlev - 2; l >= 0; --l) {
      const int Dl = D >> l, Hl = H >> l, Wl = W >> l;
      const void *below = l == nlev - 2 ? (const void *)b.e[l + 1] : (const void *)b.d[l + 1];
      CKS_FWD(conv(layers[index('d', l, true)], below, b.e[l], items, Dl, Hl, Wl, b.da[l], nullptr, s));
      CKS_FWD(conv(layers[index('d', l, false)], b.da[l], nullptr, items, Dl, Hl, Wl, b.d[l], nullptr, s));
    }
    // the head: its prediction channel alone, FP32 [V]
    const Layer &L = layers[index('h', 0, false)];
    return qesb_conv3d_head(b.d[0], L.c1, items, D, H, W, L.Bm, L.Kp, L.cout, b.y, L.bias, L.relu, d_err, s);
  }

  qesb_status ensure_scales(int n)
  {
    if (n <= nscale) return QESB_OK;
    void *p = nullptr;
    CKS_FWD(alloc(&p, sizeof(unsigned) * n));
    d_scale = static_cast<unsigned *>(p);  // the old array stays owned until release
    nscale = n;
    return QESB_OK;
  }

  void release()
  {
    cudaSetDevice(device);
    if (ev) cudaEventDestroy(ev);
    ev = nullptr;
    for (void *p : owned) cudaFree(p);
    owned.clear();
    if (h_err) cudaFreeHost(h_err);
    h_err = h_err_dev = nullptr;
    bufs.clear();
  }
};

namespace {

struct File {
  FILE *f;
  explicit File(const char *path) : f(std::fopen(path, "rb")) {}
  ~File()
  {
    if (f) std::fclose(f);
  }
  bool read(void *p, size_t bytes) { return std::fread(p, 1, bytes, f) == bytes; }
};

}  // namespace

extern "C" {

qesb_status qesb_warmnet_load(const char *path, int device, qesb_warmnet **out)
{
  if (!path || !out) return qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: null argument");
  *out = nullptr;
  File F(path);
  if (!F.f) return qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: cannot open %s", path);
  char magic[8];
  int32_t hdr[4];
  if (!F.read(magic, 8) || std::memcmp(magic, "QESBWNT1", 8) != 0 || !F.read(hdr, sizeof hdr))
    return qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: %s is not a warm-start network file", path);
  const int nlev = hdr[0], res = hdr[1];
  if (nlev < 2 || nlev > 8 || (res != 1 && res != 2) || hdr[2] != kInCh || hdr[3] != kHeadN)
    return qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: unsupported network (levels %d, res %d)", nlev, res);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return qesb_fail(QESB_ERR_NODEV, "qesb_warmnet_load: no CUDA device %d", device);
  if (cudaSetDevice(device) != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_warmnet_load: cudaSetDevice");
  auto *net = new qesb_warmnet();
  net->device = device;
  net->nlev = nlev;
  net->res = res;
  net->ch.resize(nlev);
  auto fail = [&](qesb_status s) {
    net->release();
    delete net;
    return s;
  };
  if (!F.read(net->ch.data(), sizeof(int32_t) * nlev)) return fail(qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: truncated"));
  const int nlayers = 2 * nlev + 2 * (nlev - 1) + 1;
  net->layers.resize(nlayers);
  void *p = nullptr;
  qesb_status s = QESB_OK;
  for (int q = 0; q < nlayers; ++q) {
    int32_t d[6];
    if (!F.read(d, sizeof d)) return fail(qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: truncated at layer %d", q));
    Layer &L = net->layers[q];
    L.c1 = d[0], L.c2 = d[1], L.cout = d[2], L.cout_real = d[3], L.relu = d[4], L.up1 = d[5];
    const int cin = L.c1 + L.c2;
    if (L.c1 <= 0 || L.c1 % 16 || L.c2 < 0 || L.c2 % 16 || L.cout_real < 1 || L.cout_real > L.cout ||
        (L.cout != 16 && L.cout != 32 && L.cout != 64 && L.cout != 128))
      return fail(qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: layer %d has an unsupported shape", q));
    L.Kp = (27 * cin + 63) / 64 * 64;
    std::vector<float> W((size_t)27 * cin * L.cout), b(L.cout);
    if (!F.read(W.data(), W.size() * 4) || !F.read(b.data(), b.size() * 4))
      return fail(qesb_fail(QESB_ERR_ARG, "qesb_warmnet_load: truncated at layer %d", q));
    // the tensor-core weight layout: Bm[n][k] = W[k][n], k = tap * cin + c,
    // zero beyond 27 cin and for output channels past cout_real
    std::vector<uint16_t> Bm((size_t)L.cout * L.Kp, 0);
    for (size_t row = 0; row < (size_t)27 * cin; ++row)
      for (int n = 0; n < L.cout; ++n)
        Bm[(size_t)n * L.Kp + row] = bf16_rn(n < L.cout_real ? W[row * L.cout + n] : 0.0f);
    if ((s = net->alloc(&p, Bm.size() * 2)) != QESB_OK) return fail(s);
    L.Bm = static_cast<uint16_t *>(p);
    if ((s = net->alloc(&p, b.size() * 4)) != QESB_OK) return fail(s);
    L.bias = static_cast<float *>(p);
    if (cudaMemcpy(L.Bm, Bm.data(), Bm.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(L.bias, b.data(), b.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(qesb_fail(QESB_ERR_CUDA, "qesb_warmnet_load: weight upload"));
  }
  if ((s = net->alloc(&p, sizeof(int))) != QESB_OK) return fail(s);
  net->d_err = static_cast<int *>(p);
  if (cudaHostAlloc((void **)&net->h_err, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&net->h_err_dev, net->h_err, 0) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "qesb_warmnet_load: mapped host memory"));
  if ((s = net->ensure_scales(1)) != QESB_OK) return fail(s);
  if (cudaEventCreateWithFlags(&net->ev, cudaEventDisableTiming) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "qesb_warmnet_load: cudaEventCreate"));
  *out = net;
  return QESB_OK;
}

qesb_status qesb_warmnet_destroy(qesb_warmnet *net)
{
  if (!net) return QESB_OK;
  net->release();
  delete net;
  return QESB_OK;
}

qesb_status qesb_warm_start_batch(qesb_handle *const *hs, int n, qesb_warmnet *net)
{
  if (!hs || n < 1 || !net) return qesb_fail(QESB_ERR_ARG, "qesb_warm_start: null argument");
  int Nx = 0, Ny = 0, Nz = 0, dev = -1;
  for (int i = 0; i < n; ++i) {
    if (!hs[i]) return qesb_fail(QESB_ERR_ARG, "qesb_warm_start: null handle %d", i);
    int x = 0, y = 0, z = 0, d = -1;
    CKS_FWD(qesb_handle_grid(hs[i], &x, &y, &z, &d));
    if (i == 0) {
      Nx = x, Ny = y, Nz = z, dev = d;
    } else if (x != Nx || y != Ny || z != Nz || d != dev) {
      return qesb_fail(QESB_ERR_ARG, "qesb_warm_start: handle %d's grid or device differs from handle 0's", i);
    }
  }
  if (dev != net->device)
    return qesb_fail(QESB_ERR_ARG, "qesb_warm_start: network on device %d, handle on device %d", net->device, dev);
  const int F = net->res << (net->nlev - 1);
  if (Nx % F || Ny % F || Nz % F)
    return qesb_fail(QESB_ERR_ARG, "qesb_warm_start: grid %d x %d x %d not divisible by %d", Nx, Ny, Nz, F);
  std::lock_guard<std::mutex> lk(net->mu);
  if (cudaSetDevice(net->device) != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_warm_start: cudaSetDevice");
  std::vector<void *> st(n);
  for (int i = 0; i < n; ++i) CKS_FWD(qesb_get_stream(hs[i], &st[i]));
  void *s = st[0];
  const int D = Nz / net->res, H = Ny / net->res, W = Nx / net->res;
  const size_t V0 = (size_t)D * H * W;
  Buffers *b = nullptr;
  CKS_FWD(net->buffers(n * D, H, W, &b));
  CKS_FWD(net->ensure_scales(n));
  auto join = [&](void *from, void *to) -> qesb_status {  // work on `to` after what `from` holds so far
    if (from == to) return QESB_OK;
    if (cudaEventRecord(net->ev, (cudaStream_t)from) != cudaSuccess ||
        cudaStreamWaitEvent((cudaStream_t)to, net->ev, 0) != cudaSuccess)
      return qesb_fail(QESB_ERR_CUDA, "qesb_warm_start: stream ordering");
    return QESB_OK;
  };
  for (int i = 0; i < n; ++i) {  // each item's input on its handle's stream, then ordered before the forward
    uint16_t *x = b->x + V0 * kInCh * i;
    CKS_FWD(join(s, st[i]));
    CKS_FWD(qesb_compute_divergence(hs[i]));
    if (net->res == 1) CKS_FWD(qesb_warm_input(hs[i], x, kInCh, net->d_scale + i));
    else CKS_FWD(qesb_warm_input_half(hs[i], x, kInCh, net->d_scale + i));
    CKS_FWD(join(st[i], s));
  }
  CKS_FWD(net->forward(*b, n, D, H, W, s));
  for (int i = 0; i < n; ++i) {
    const float *y = b->y + V0 * i;
    CKS_FWD(join(s, st[i]));
    CKS_FWD(net->res == 1 ? qesb_warm_apply(hs[i], y, 1, net->d_scale + i)
                          : qesb_warm_apply_up2(hs[i], y, 1, net->d_scale + i));
  }
  // the error flag through mapped memory (a copy would queue behind other streams' transfers)
  CKS_FWD(qesb_copy_small(net->h_err_dev, net->d_err, sizeof(int), s));
  if (cudaStreamSynchronize((cudaStream_t)s) != cudaSuccess)
    return qesb_fail(QESB_ERR_CUDA, "qesb_warm_start: %s", cudaGetErrorString(cudaGetLastError()));
  const int err = *net->h_err;
  for (int i = 0; i < n; ++i)
    if (st[i] != s && cudaStreamSynchronize((cudaStream_t)st[i]) != cudaSuccess)
      return qesb_fail(QESB_ERR_CUDA, "qesb_warm_start: %s", cudaGetErrorString(cudaGetLastError()));
  if (err) return qesb_fail(QESB_ERR_CUDA, "qesb_warm_start: a tensor-core completion wait gave up");
  return QESB_OK;
}

qesb_status qesb_warm_start(qesb_handle *h, qesb_warmnet *net) { return qesb_warm_start_batch(&h, 1, net); }

}  // extern "C"
