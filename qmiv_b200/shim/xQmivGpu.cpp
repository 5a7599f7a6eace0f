// Drop-in adapter for a QMIV host, see xQmivGpu.h.
#include "xQmivGpu.h"

#include <limits>

namespace PMBB_NAMESPACE {

qmiv_status xQmivGpu::create(int32 Device, int32V2 Size, int32 BitDepth, const qmiv_params* Params)
{
  destroy();
  qmiv_status s = qmiv_ctx_create(Device, 0, &m_Ctx);
  if(s != QMIV_OK) { m_Ctx = nullptr; return s; }
  // the app's pictures are 4:4:4 (xSeqPic::xUnpackFrame upsamples 4:2:0 / 4:2:2 chroma on reading)
  s = qmiv_calc_create(m_Ctx, Size.getX(), Size.getY(), BitDepth, 444, Params, &m_Calc);
  if(s != QMIV_OK) { m_Calc = nullptr; destroy(); return s; }
  m_Size = Size;
  m_BitDepth = BitDepth;
  return QMIV_OK;
}

void xQmivGpu::destroy()
{
  if(m_Calc) { qmiv_calc_destroy(m_Calc); m_Calc = nullptr; }
  if(m_Ctx) { qmiv_ctx_destroy(m_Ctx); m_Ctx = nullptr; }
  for(std::vector<uint8>& p : m_Packed) { std::vector<uint8>().swap(p); }
}

// A host frame over the picture's three components. Pictures above 8 bits are used in place (uint16
// samples from each component's origin, row pitch = stride); 8-bit pictures are packed to bytes.
qmiv_status xQmivGpu::xBindFrame(const xPicP* Pic, int32 Slot, qmiv_frame* Frame)
{
  if(Pic == nullptr || Pic->getWidth() != m_Size.getX() || Pic->getHeight() != m_Size.getY() ||
     Pic->getBitDepth() != m_BitDepth)
  {
    return QMIV_ERR_INVALID_ARG;
  }
  const int32 W = m_Size.getX(), H = m_Size.getY(), Stride = Pic->getStride();
  Frame->mem = QMIV_MEM_HOST;
  if(m_BitDepth > 8)
  {
    for(int32 c = 0; c < 3; c++)
    {
      Frame->plane[c] = Pic->getAddr((eCmp)c);
      Frame->pitch[c] = (int64_t)Stride * (int64_t)sizeof(uint16);
    }
    return QMIV_OK;
  }
  std::vector<uint8>& Buf = m_Packed[Slot];
  Buf.resize((size_t)3 * W * H);
  for(int32 c = 0; c < 3; c++)
  {
    const uint16* Src = Pic->getAddr((eCmp)c);
    uint8* Dst = Buf.data() + (size_t)c * W * H;
    for(int32 y = 0; y < H; y++)
    {
      for(int32 x = 0; x < W; x++) { Dst[(size_t)y * W + x] = (uint8)Src[(size_t)y * Stride + x]; }
    }
    Frame->plane[c] = Dst;
    Frame->pitch[c] = W;
  }
  return QMIV_OK;
}

qmiv_status xQmivGpu::calcFrame(const xPicP* Pic0, const xPicP* Pic1, uint32 MetricMask, qmiv_result* Result)
{
  if(m_Calc == nullptr || Result == nullptr) { return QMIV_ERR_INVALID_ARG; }
  qmiv_frame F0, F1;
  qmiv_status s = xBindFrame(Pic0, 0, &F0);
  if(s == QMIV_OK) { s = xBindFrame(Pic1, 1, &F1); }
  if(s != QMIV_OK) { return s; }
  return qmiv_frame_pair_compute(m_Calc, &F0, &F1, MetricMask, Result);
}

namespace {
constexpr flt64 kNaN = std::numeric_limits<flt64>::quiet_NaN();
}

flt64V4 xQmivGpu::calcPicPSNR(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_PSNR, &R) == QMIV_OK ? flt64V4(R.psnr) : flt64V4(kNaN, kNaN, kNaN, kNaN);
}

flt64V4 xQmivGpu::calcPicWSPSNR(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_WSPSNR, &R) == QMIV_OK ? flt64V4(R.wspsnr) : flt64V4(kNaN, kNaN, kNaN, kNaN);
}

flt64 xQmivGpu::calcPicIVPSNR(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_IVPSNR, &R) == QMIV_OK ? R.ivpsnr : kNaN;
}

flt64V4 xQmivGpu::calcPicSSIM(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_SSIM, &R) == QMIV_OK ? flt64V4(R.ssim) : flt64V4(kNaN, kNaN, kNaN, kNaN);
}

flt64V4 xQmivGpu::calcPicMSSSIM(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_MSSSIM, &R) == QMIV_OK ? flt64V4(R.msssim) : flt64V4(kNaN, kNaN, kNaN, kNaN);
}

flt64 xQmivGpu::calcPicIVSSIM(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_IVSSIM, &R) == QMIV_OK ? R.ivssim : kNaN;
}

flt64 xQmivGpu::calcPicIVMSSSIM(const xPicP* Pic0, const xPicP* Pic1)
{
  qmiv_result R{};
  return calcFrame(Pic0, Pic1, QMIV_IVMSSSIM, &R) == QMIV_OK ? R.ivmsssim : kNaN;
}

} // end of namespace PMBB_NAMESPACE
