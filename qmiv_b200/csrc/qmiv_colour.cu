// Colour-space conversion before the metrics: the app's -csi / -csm options
// (apps/QMIV/src/xAppQMIV.cpp:302-311 choose the conversion, :853-891 run it on the 4:4:4 pictures
// before the exactness check and every metric). One kernel reads both frames in their own chroma
// format (chroma sample (x >> sx, y >> sy)), applies the invalid-sample check and conceal the
// reference runs before it (:834-852), converts each 4:4:4 pixel with the integer fixed-point
// matrices the reference dispatches to (libs/pmbb-core/src/xColorSpaceSTD.cpp:196-263 and their SIMD
// forms) or reorders BGR / GBR to RGB, and writes 4:4:4 planes of the picture's sample type. The
// frame pipeline then runs on those planes with a 4:4:4 shape.
#include "qmiv_host.h"

#include <cstring>

namespace qmiv {

namespace {

// 16 fractional bits; rows as the reference's xColorSpaceCoeffYCbCr integer matrices
// (xColorSpaceCoeff.h:59-73), which the results must round like: BT.601 (= SMPTE 170M), BT.709,
// SMPTE 240M, BT.2020. RGB -> YCbCr: (Y<-R, Y<-G, Y<-B, Cb<-R, Cb<-G, Cr<-G, Cr<-B), the Cb<-B and
// Cr<-R entries being 1/2. YCbCr -> RGB: (R<-Cr, G<-Cb, G<-Cr, B<-Cb), the Y entries being 1.
__constant__ int32_t c_rgb2ycc[4][7] = {
  { 19595, 38470, 7471, -11058, -21710, -27439, -5329 },
  { 13933, 46871, 4732, -7509, -25259, -29763, -3005 },
  { 13894, 45941, 5701, -7609, -25159, -29150, -3618 },
  { 17216, 44434, 3886, -9151, -23617, -30133, -2635 },
};
__constant__ int32_t c_ycc2rgb[4][4] = {
  { 91881, -22553, -46802, 116130 },
  { 103206, -12276, -30679, 121609 },
  { 103285, -14852, -31236, 119669 },
  { 96639, -10784, -37444, 123299 },
};

struct ColourArgs
{
  Img      in[2];
  MutImg   out[2];             // 4:4:4 planes, pitch W
  int32_t  W, H;
  uint32_t clip;               // conceal: samples above are clipped (65535 = no clipping)
  int32_t  mode;               // 0 none, 1 YCbCr -> RGB, 2 RGB -> YCbCr
  int32_t  space;              // matrix index 0..3
  int32_t  perm[3];            // output component k takes converted component perm[k]
  int32_t  bitdepth;
  uint32_t* max_sample;        // [2]
};

__device__ __forceinline__ int32_t clip_u(int32_t v, int32_t mx) { return min(max(v, 0), mx); }
// products and sums in two's complement like the reference's int32 arithmetic
__device__ __forceinline__ int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

template <typename T>
__global__ void __launch_bounds__(256) k_colour(const __grid_constant__ ColourArgs a)
{
  const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int f = blockIdx.z;
  uint32_t mx = 0;
  if(x < a.W && y < a.H)
  {
    int32_t v[3];
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const uint32_t s = (uint32_t)fetch<T>(a.in[f], c, x, y);
      mx = max(mx, s);
      v[c] = (int32_t)min(s, a.clip);
    }
    const int32_t maxv = (1 << a.bitdepth) - 1, mid = 1 << (a.bitdepth - 1), add = 1 << 15;
    int32_t o[3] = { v[0], v[1], v[2] };
    if(a.mode == 1)                                           // xColorSpaceSTD.cpp:231-263
    {
      const int32_t* k = c_ycc2rgb[a.space];
      const int32_t iu = v[1] - mid, iv = v[2] - mid;
      const int32_t sy = wadd((int32_t)((uint32_t)v[0] << 16), add);
      o[0] = clip_u(wadd(sy, wmul(k[0], iv)) >> 16, maxv);
      o[1] = clip_u(wadd(wadd(sy, wmul(k[1], iu)), wmul(k[2], iv)) >> 16, maxv);
      o[2] = clip_u(wadd(sy, wmul(k[3], iu)) >> 16, maxv);
    }
    else if(a.mode == 2)                                      // xColorSpaceSTD.cpp:196-229
    {
      const int32_t* k = c_rgb2ycc[a.space];
      const int32_t r = v[0], g = v[1], b = v[2];
      const int32_t ty = wadd(wadd(wadd(wmul(k[0], r), wmul(k[1], g)), wmul(k[2], b)), add) >> 16;
      const int32_t tu = wadd(wadd(wadd(wmul(k[3], r), wmul(k[4], g)), (int32_t)((uint32_t)b << 15)), add) >> 16;
      const int32_t tv = wadd(wadd(wadd((int32_t)((uint32_t)r << 15), wmul(k[5], g)), wmul(k[6], b)), add) >> 16;
      o[0] = clip_u(ty, maxv);
      o[1] = clip_u(tu + mid, maxv);
      o[2] = clip_u(tv + mid, maxv);
    }
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const int32_t val = a.perm[c] == 0 ? o[0] : (a.perm[c] == 1 ? o[1] : o[2]);
      static_cast<T*>(a.out[f].p[c])[(size_t)y * a.out[f].pitch[c] + x] = (T)val;
    }
  }
  mx = __reduce_max_sync(0xffffffffu, mx);
  if((threadIdx.x & 31) == 0 && mx) { atomicMax(a.max_sample + f, mx); }
}

bool cs_is_rgb(int32_t c) { return c == QMIV_CS_RGB || c == QMIV_CS_BGR || c == QMIV_CS_GBR; }
bool cs_is_defined_ycc(int32_t c) { return c > QMIV_CS_YCBCR && c <= QMIV_CS_BT2020; }
int  cs_index(int32_t c)
{
  switch(c)
  {
  case QMIV_CS_BT601: case QMIV_CS_SMPTE170M: return 0;
  case QMIV_CS_BT709: return 1;
  case QMIV_CS_SMPTE240M: return 2;
  case QMIV_CS_BT2020: return 3;
  default: return -1;
  }
}

}  // namespace

// The app's checks of the two options (xAppQMIV.cpp:299-306) and the conversion they select (:308-310).
qmiv_status ColourStage::configure(int32_t cs_in, int32_t cs_metric)
{
  auto known = [](int32_t c) { return cs_is_rgb(c) || c == QMIV_CS_YCBCR || cs_is_defined_ycc(c); };
  if(!known(cs_in) || !known(cs_metric)) { return fail(QMIV_ERR_INVALID_ARG, "unknown colour space"); }
  if(cs_in != cs_metric)
  {
    if(cs_in >= QMIV_CS_YCBCR && cs_metric >= QMIV_CS_YCBCR) { return fail(QMIV_ERR_UNSUPPORTED, "YCbCr to YCbCr conversion is not supported"); }
    if(cs_in == QMIV_CS_YCBCR || cs_metric == QMIV_CS_YCBCR) { return fail(QMIV_ERR_INVALID_ARG, "generic YCbCr cannot be used for conversion"); }
  }
  mode = 0; space = 0; perm[0] = 0; perm[1] = 1; perm[2] = 2;
  if(cs_is_defined_ycc(cs_in) && cs_is_rgb(cs_metric)) { mode = 1; space = cs_index(cs_in); }
  if(cs_is_rgb(cs_in) && cs_is_defined_ycc(cs_metric)) { mode = 2; space = cs_index(cs_metric); }
  if(cs_is_rgb(cs_in) && cs_in != QMIV_CS_RGB && cs_metric == QMIV_CS_RGB)
  {
    // BGR -> RGB swaps components 0 and 2; GBR -> RGB swaps 0 and 1, then 0 and 2 (xAppQMIV.cpp:878-891)
    if(cs_in == QMIV_CS_BGR) { perm[0] = 2; perm[1] = 1; perm[2] = 0; }
    if(cs_in == QMIV_CS_GBR) { perm[0] = 2; perm[1] = 0; perm[2] = 1; }
  }
  active = mode != 0 || perm[0] != 0 || perm[1] != 1;
  return QMIV_OK;
}

ColourStage::~ColourStage()
{
  if(h_max_) { cudaFreeHost(h_max_); }
}

qmiv_status ColourStage::convert(qmiv_ctx_s* ctx, const Shape& S, const qmiv_params& prm, const Img& in0, const Img& in1, Img& out0,
                                 Img& out1, cudaStream_t s)
{
  if(!configured_ || !(shape444_.W == S.W && shape444_.H == S.H && shape444_.bitdepth == S.bitdepth))
  {
    QMIV_TRY(shape444_.init(S.W, S.H, S.bitdepth, 444));
    QMIV_TRY(pipe444.configure(ctx, shape444_, prm, prm.search_range));
    configured_ = true;
  }
  const size_t plane = (size_t)S.W * S.H * S.esz;
  QMIV_TRY(planes_.ensure(ctx, 6 * plane));
  QMIV_TRY(max_.ensure(ctx, 2 * sizeof(uint32_t)));
  if(!h_max_) { QMIV_CUDA(cudaMallocHost((void**)&h_max_, 2 * sizeof(uint32_t))); }
  ColourArgs a{};
  a.in[0] = in0; a.in[1] = in1;
  Img* outs[2] = { &out0, &out1 };
  for(int f = 0; f < 2; f++)
  {
    *outs[f] = Img{};
    for(int c = 0; c < 3; c++)
    {
      void* p = planes_.as<char>() + (size_t)(3 * f + c) * plane;
      a.out[f].p[c] = p; a.out[f].pitch[c] = S.W;
      outs[f]->p[c] = p; outs[f]->pitch[c] = S.W; outs[f]->sx[c] = 0; outs[f]->sy[c] = 0;
    }
  }
  a.W = S.W; a.H = S.H;
  a.clip = prm.invalid_pel_action == QMIV_PEL_CNCL ? (uint32_t)S.maxv : 0xffffu;
  a.mode = mode; a.space = space < 0 ? 0 : space;
  for(int c = 0; c < 3; c++) { a.perm[c] = perm[c]; }
  a.bitdepth = S.bitdepth;
  a.max_sample = max_.as<uint32_t>();
  QMIV_CUDA(cudaMemsetAsync(max_.p, 0, 2 * sizeof(uint32_t), s));
  const dim3 grid((S.W + 31) / 32, (S.H + 7) / 8, 2);
  if(S.esz == 1) { k_colour<uint8_t><<<grid, 256, 0, s>>>(a); }
  else { k_colour<uint16_t><<<grid, 256, 0, s>>>(a); }
  QMIV_CUDA(cudaGetLastError());
  QMIV_CUDA(cudaMemcpyAsync(h_max_, max_.p, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  return QMIV_OK;
}

int32_t ColourStage::invalid_flags(int32_t maxv) const
{
  return (h_max_ && h_max_[0] > (uint32_t)maxv ? 1 : 0) | (h_max_ && h_max_[1] > (uint32_t)maxv ? 2 : 0);
}

}  // namespace qmiv
