// slab_fft.cu -- a 3-D real FFT of one grid split over P GPUs (one process per GPU) in
// z slabs: the pieces a driver composes around its all-to-all (NCCL over NVLink).  This
// is the reference's P3DFFT decomposition (Multi_MEUMAPPS.f:124-128 sets up the process
// grid, :241-248 the P3DFFT plan; f_trans / inv_trans at ModFunc.f:15-40) for grids
// larger than one GPU holds, with one exchange per transform instead of P3DFFT's two.
//
// Rank r holds the real z-planes [r*NZL, (r+1)*NZL) as [z][y][x] (NZL = Nz/P) and, after
// the forward transform, the spectrum of the ky rows [r*NYL, (r+1)*NYL) as [kz][ky][kx]
// (NYL = Ny/P, kx in [0, Nx/2]).  Forward:
//   planes : x R2C and y FFT of the rank's planes, then PACK into P chunks, chunk d =
//            [z][ky in d's rows][kx] scaled by 1/P (send buffer [P][NZL][NYL][NXH])
//   (caller: all-to-all of equal chunks; chunk q received from rank q lands at
//            [q][NZL][NYL][NXH], which is the k-slab [kz][ky][kx] in z order)
//   columns: z FFT of the k-slab in place, scaled by 1/(Nx NYL Nz) -- with the pack's
//            1/P the f_trans scale 1/(Nx Ny Nz)
// Inverse: columns (z iFFT in place; chunk q of the k-slab = its kz rows of rank q's
// planes), all-to-all, then planes (UNPACK chunk d into the d rows of ky, y iFFT, x C2R).
#include <memory>
#include <string>

#include "../../include/meu.h"
#include "fft.cuh"

namespace meu {

// send[d][z][y'][kx] = s * spec[z][d*NYL + y'][kx]
template <typename C, typename R>
__global__ void k_slab_pack(const C* __restrict__ spec, C* __restrict__ send, int P, int nzl, int ny, int nyl, int nxh,
                            R s) {
  const int64_t total = (int64_t)P * nzl * nyl * nxh;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(i % nxh);
    int64_t t = i / nxh;
    const int yp = (int)(t % nyl);
    t /= nyl;
    const int z = (int)(t % nzl);
    const int d = (int)(t / nzl);
    const C v = spec[((int64_t)z * ny + (int64_t)d * nyl + yp) * nxh + kx];
    send[i] = cscale(v, s);
  }
}
// spec[z][d*NYL + y'][kx] = recv[d][z][y'][kx]
template <typename C>
__global__ void k_slab_unpack(const C* __restrict__ recv, C* __restrict__ spec, int P, int nzl, int ny, int nyl,
                              int nxh) {
  const int64_t total = (int64_t)P * nzl * nyl * nxh;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(i % nxh);
    int64_t t = i / nxh;
    const int yp = (int)(t % nyl);
    t /= nyl;
    const int z = (int)(t % nzl);
    const int d = (int)(t / nzl);
    spec[((int64_t)z * ny + (int64_t)d * nyl + yp) * nxh + kx] = recv[i];
  }
}

}  // namespace meu

struct meu_slab_fft {
  int nx = 0, ny = 0, nz = 0, P = 1, rank = 0, nzl = 0, nyl = 0, nxh = 0;
  bool f64 = false;
  std::unique_ptr<meu::FFT3> planes;  // (Nx, Ny, NZL): x and y passes of the rank's planes
  std::unique_ptr<meu::FFT3> cols;    // (Nx, NYL, Nz): z pass of the rank's k-slab
  void* spec = nullptr;               // [NZL][Ny][NXH] complex: the planes' spectrum
  int64_t launches = 0;
  std::string err;
  ~meu_slab_fft() {
    if (spec) cudaFree(spec);
  }
};

namespace {
using namespace meu;

int fail(meu_slab_fft* h, const std::string& m, int code) {
  if (h) h->err = m;
  set_thread_error(m);
  return code;
}

template <typename R>
void planes_forward(meu_slab_fft* h, const void* real, void* send, cudaStream_t st) {
  using C = cplx<R>;
  PtrList<const R> a{};
  PtrList<C> b{};
  a.p[0] = (const R*)real;
  b.p[0] = (C*)h->spec;
  h->planes->forward_x<R>(a, b, 1, st);
  h->planes->pass_y<R>(b, 1, true, st);
  const int64_t n = (int64_t)h->P * h->nzl * h->nyl * h->nxh;
  k_slab_pack<C, R><<<grid_for(n, 256), 256, 0, st>>>((const C*)h->spec, (C*)send, h->P, h->nzl, h->ny, h->nyl,
                                                       h->nxh, (R)(1.0 / h->P));
  MEU_CHECK_LAUNCH();
  h->launches += 3;
}
template <typename R>
void planes_inverse(meu_slab_fft* h, const void* recv, void* real, cudaStream_t st) {
  using C = cplx<R>;
  const int64_t n = (int64_t)h->P * h->nzl * h->nyl * h->nxh;
  k_slab_unpack<C><<<grid_for(n, 256), 256, 0, st>>>((const C*)recv, (C*)h->spec, h->P, h->nzl, h->ny, h->nyl,
                                                     h->nxh);
  MEU_CHECK_LAUNCH();
  PtrList<C> b{};
  PtrList<R> o{};
  b.p[0] = (C*)h->spec;
  o.p[0] = (R*)real;
  h->planes->pass_y<R>(b, 1, false, st);
  h->planes->inverse_x<R>(b, o, 1, st);
  h->launches += 3;
}
template <typename R>
void columns(meu_slab_fft* h, void* kslab, bool fwd, cudaStream_t st) {
  PtrList<cplx<R>> b{};
  b.p[0] = (cplx<R>*)kslab;
  h->cols->pass_z<R>(b, 1, fwd, st);
  h->launches += 1;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }
}  // namespace

#define MEU_SLAB_TRY(h, name, body)                                         \
  try {                                                                     \
    body;                                                                   \
  } catch (const meu::CudaError& e) {                                       \
    return fail(h, std::string(name ": ") + e.what(), e.code);              \
  } catch (const std::bad_alloc&) {                                         \
    return fail(h, name ": host allocation failed", MEU_ERR_NOMEM);         \
  } catch (const std::exception& e) {                                       \
    return fail(h, std::string(name ": ") + e.what(), MEU_ERR_CUDA);        \
  }                                                                         \
  return MEU_OK;

extern "C" int meu_slab_fft_create(int32_t nx, int32_t ny, int32_t nz, int32_t nranks, int32_t rank,
                                   int32_t precision, meu_slab_fft** out) {
  if (!out) return fail(nullptr, "meu_slab_fft_create: NULL handle pointer", MEU_ERR_BADARG);
  *out = nullptr;
  if (precision != MEU_PREC_F64 && precision != MEU_PREC_F32)
    return fail(nullptr, "meu_slab_fft_create: unknown precision", MEU_ERR_BADARG);
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return fail(nullptr, "meu_slab_fft_create: rank outside [0, nranks)", MEU_ERR_BADARG);
  if (nz % nranks != 0 || ny % nranks != 0)
    return fail(nullptr, "meu_slab_fft_create: Ny and Nz must be multiples of the rank count", MEU_ERR_BADARG);
  const int nzl = nz / nranks, nyl = ny / nranks;
  if (!fft_size_ok(nx, true) || !fft_size_ok(ny, false) || !fft_size_ok(nz, false) || !fft_size_ok(nzl, false) ||
      !fft_size_ok(nyl, false))
    return fail(nullptr, "meu_slab_fft_create: Nx, Ny, Nz, Ny/P and Nz/P must be 2^a 3^b (Nx even)",
                MEU_ERR_UNSUPPORTED);
  std::unique_ptr<meu_slab_fft> h(new meu_slab_fft);
  MEU_SLAB_TRY(nullptr, "meu_slab_fft_create", {
    h->nx = nx;
    h->ny = ny;
    h->nz = nz;
    h->P = nranks;
    h->rank = rank;
    h->nzl = nzl;
    h->nyl = nyl;
    h->nxh = nx / 2 + 1;
    h->f64 = precision == MEU_PREC_F64;
    h->planes.reset(new FFT3(nx, ny, nzl, h->f64));
    h->cols.reset(new FFT3(nx, nyl, nz, h->f64));
    const size_t cb = h->f64 ? sizeof(double2) : sizeof(float2);
    MEU_CUDA(cudaMalloc(&h->spec, cb * (size_t)nzl * ny * h->nxh));
    *out = h.release();
  })
}

/* out4: real slab elements (NZL*Ny*Nx), one chunk's complex elements (NZL*NYL*NXH),
 * the send / receive / k-slab buffer's complex elements (P chunks = Nz*NYL*NXH), P */
extern "C" int meu_slab_fft_sizes(const meu_slab_fft* h, int64_t* out4) {
  if (!h || !out4) return fail(nullptr, "meu_slab_fft_sizes: NULL argument", MEU_ERR_BADARG);
  out4[0] = (int64_t)h->nzl * h->ny * h->nx;
  out4[1] = (int64_t)h->nzl * h->nyl * h->nxh;
  out4[2] = (int64_t)h->P * out4[1];
  out4[3] = h->P;
  return MEU_OK;
}

extern "C" int meu_slab_fft_forward_planes(meu_slab_fft* h, const void* real_dev, void* send_dev, void* stream) {
  if (!h || !real_dev || !send_dev) return fail(h, "meu_slab_fft_forward_planes: NULL argument", MEU_ERR_BADARG);
  if (!aligned16(real_dev) || !aligned16(send_dev))
    return fail(h, "meu_slab_fft_forward_planes: device arrays must be 16-byte aligned", MEU_ERR_BADARG);
  MEU_SLAB_TRY(h, "meu_slab_fft_forward_planes", {
    if (h->f64) planes_forward<double>(h, real_dev, send_dev, (cudaStream_t)stream);
    else planes_forward<float>(h, real_dev, send_dev, (cudaStream_t)stream);
  })
}

extern "C" int meu_slab_fft_forward_columns(meu_slab_fft* h, void* kslab_dev, void* stream) {
  if (!h || !kslab_dev) return fail(h, "meu_slab_fft_forward_columns: NULL argument", MEU_ERR_BADARG);
  if (!aligned16(kslab_dev))
    return fail(h, "meu_slab_fft_forward_columns: device array must be 16-byte aligned", MEU_ERR_BADARG);
  MEU_SLAB_TRY(h, "meu_slab_fft_forward_columns", {
    if (h->f64) columns<double>(h, kslab_dev, true, (cudaStream_t)stream);
    else columns<float>(h, kslab_dev, true, (cudaStream_t)stream);
  })
}

extern "C" int meu_slab_fft_inverse_columns(meu_slab_fft* h, void* kslab_dev, void* stream) {
  if (!h || !kslab_dev) return fail(h, "meu_slab_fft_inverse_columns: NULL argument", MEU_ERR_BADARG);
  if (!aligned16(kslab_dev))
    return fail(h, "meu_slab_fft_inverse_columns: device array must be 16-byte aligned", MEU_ERR_BADARG);
  MEU_SLAB_TRY(h, "meu_slab_fft_inverse_columns", {
    if (h->f64) columns<double>(h, kslab_dev, false, (cudaStream_t)stream);
    else columns<float>(h, kslab_dev, false, (cudaStream_t)stream);
  })
}

extern "C" int meu_slab_fft_inverse_planes(meu_slab_fft* h, const void* recv_dev, void* real_dev, void* stream) {
  if (!h || !recv_dev || !real_dev) return fail(h, "meu_slab_fft_inverse_planes: NULL argument", MEU_ERR_BADARG);
  if (!aligned16(recv_dev) || !aligned16(real_dev))
    return fail(h, "meu_slab_fft_inverse_planes: device arrays must be 16-byte aligned", MEU_ERR_BADARG);
  MEU_SLAB_TRY(h, "meu_slab_fft_inverse_planes", {
    if (h->f64) planes_inverse<double>(h, recv_dev, real_dev, (cudaStream_t)stream);
    else planes_inverse<float>(h, recv_dev, real_dev, (cudaStream_t)stream);
  })
}

extern "C" int64_t meu_slab_fft_launch_count(const meu_slab_fft* h) { return h ? h->launches : 0; }

extern "C" const char* meu_slab_fft_last_error(const meu_slab_fft* h) { return h ? h->err.c_str() : ""; }

extern "C" int meu_slab_fft_destroy(meu_slab_fft* h) {
  delete h;
  return MEU_OK;
}
