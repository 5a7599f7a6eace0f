/*
  C-ABI shim around the QMIV reference library (pmbb-base/core/ivqm), compiled
  together with the reference's own sources by oracle/Makefile into
  oracle/_ref/<arch>/libqmivref.so.

  TEST INFRASTRUCTURE ONLY: this file is never part of the product library.
  It lets the tests and the golden-fixture generator run the unmodified
  reference algorithms on in-memory frames, following the per-frame call
  sequence of the reference app:
    apps/QMIV/src/xAppQMIV.cpp:761-827   processAllFrames (order of steps)
    apps/QMIV/src/xAppQMIV.cpp:853-907   preprocessFrames (exact flags, extend)
    apps/QMIV/src/xAppQMIV.cpp:908-917   rearrangePictures (planar -> interleaved)
    apps/QMIV/src/xAppQMIV.cpp:927-948   calcFrameGCD / calcFrameSCP
    apps/QMIV/src/xAppQMIV.cpp:967-1108  calcFrame____PSNR .. calcFrameIVMSSSIM
    apps/QMIV/src/xAppQMIV.cpp:680-744   createProcessors (parameter plumbing)
    apps/QMIV/src/xAppQMIV.cpp:900-1030  mask mode (NumNonMasked, GCD-M, PSNR-M, WS-PSNR-M, IV-PSNR-M)
    libs/pmbb-core/src/xSeq.cpp:231-290  xUnpackFrame (8->16 bit, chroma upsampling)
*/
#include "xPic.h"
#include "xPixelOps.h"
#include "xThreadPool.h"
#include "xGlobClrDiff.h"
#include "xShftCompPic.h"
#include "xCorrespPixelShift.h"
#include "xIVPSNR.h"
#include "xIVSSIM.h"
#include "xStructSim.h"
#include "xTestUtils.h"
#include "xTestUtilsIVQM.h"
#include "xKBNS.h"
#include "xColorSpace.h"
#include <cstring>
#include <cstdint>
#include <vector>

using namespace PMBB_NAMESPACE;

extern "C" {

struct ref_params
{
  int32_t width, height, bitdepth, chroma_format; /* 420, 422, 444 */
  int32_t search_range;
  int32_t cws[4];
  int32_t cwa[4];
  float   unc[4];
  int32_t erp, lon_range, lat_range;
  int32_t num_threads; /* 0 = run inline */
};

struct ref_result
{
  int32_t gcd_r2t[4];
  int32_t exact[4];
  double  psnr[4];   double psnr_pic;
  double  wspsnr[4]; double wspsnr_pic;
  double  ivpsnr;    double ivpsnr_r2t;   double ivpsnr_t2r;
  double  ssim[4];   double ssim_pic;
  double  msssim[4]; double msssim_pic;
  double  ivssim;    double ivssim_r2t;   double ivssim_t2r;
  double  ivmsssim;  double ivmsssim_r2t; double ivmsssim_t2r;
};

enum { REF_PSNR = 1, REF_WSPSNR = 2, REF_IVPSNR = 4, REF_SSIM = 8, REF_MSSSIM = 16, REF_IVSSIM = 32, REF_IVMSSSIM = 64 };

/* Structural similarity options of the app (-ssm, -ssb, -ssw, -sss; apps/QMIV/src/xAppQMIV.cpp:99-104,
   325-332): mode as xSSIM::eMode (0 RegularGaussianFlt, 1 RegularGaussianInt, 2 RegularAveraged,
   3 BlockGaussianInt, 4 BlockAveraged), border as eMrgExt (0 None .. 5 Zero). */
struct ref_ssim_cfg
{
  int32_t mode, border, window, stride;
};

} // extern "C"

namespace {

// Load one raw frame (planar Y, U, V; 1 byte per sample for bitdepth 8, else 2 bytes LE) into a planar
// 4:4:4 xPicP, mirroring xSeqPic::xUnpackFrame (xSeq.cpp:231-290).
void loadFrame(xPicP& Pic, const void* const Planes[3], int32 W, int32 H, int32 BitDepth, int32 ChromaFormat)
{
  const int32 Stride = Pic.getStride();
  const bool  Byte   = BitDepth <= 8;
  if(Byte) { xPixelOps::Cvt(Pic.getAddr(eCmp::LM), (const uint8*)Planes[0], Stride, W, W, H); }
  else     { xPixelOps::Copy(Pic.getAddr(eCmp::LM), (const uint16*)Planes[0], Stride, W, W, H); }
  for(int32 c = 1; c < 3; c++)
  {
    uint16* Dst = Pic.getAddr((eCmp)c);
    if(ChromaFormat == 420)
    {
      if(Byte) { xPixelOps::CvtUpsampleHV(Dst, (const uint8 *)Planes[c], Stride, W >> 1, W, H); }
      else     { xPixelOps::UpsampleHV   (Dst, (const uint16*)Planes[c], Stride, W >> 1, W, H); }
    }
    else if(ChromaFormat == 422)
    {
      if(Byte) { xPixelOps::CvtUpsampleH(Dst, (const uint8 *)Planes[c], Stride, W >> 1, W, H); }
      else     { xPixelOps::UpsampleH   (Dst, (const uint16*)Planes[c], Stride, W >> 1, W, H); }
    }
    else
    {
      if(Byte) { xPixelOps::Cvt (Dst, (const uint8 *)Planes[c], Stride, W, W, H); }
      else     { xPixelOps::Copy(Dst, (const uint16*)Planes[c], Stride, W, W, H); }
    }
  }
}

struct Pool
{
  xThreadPool* ThreadPool = nullptr;
  tThPI        TPI;
  explicit Pool(int32 NumThreads, int32 H)
  {
    if(NumThreads > 0)
    {
      ThreadPool = new xThreadPool;
      ThreadPool->create(NumThreads, H + 1);
      TPI.init(ThreadPool, H + 1, H + 1);
    }
  }
  ~Pool()
  {
    if(ThreadPool) { TPI.uninit(); ThreadPool->destroy(); delete ThreadPool; }
  }
};

void copyPlanar(uint16_t* Dst, const xPicP& Src, int32 W, int32 H)
{
  for(int32 c = 0; c < 3; c++)
  {
    const uint16* S = Src.getAddr((eCmp)c);
    for(int32 y = 0; y < H; y++) { std::memcpy(Dst + ((size_t)c * H + y) * W, S + (size_t)y * Src.getStride(), W * sizeof(uint16)); }
  }
}

} // namespace

extern "C" {

/* Colour spaces of the app's -csi / -csm options (apps/QMIV/src/xUtilsQMIV.h:12-27). */
enum { REF_CS_RGB = 2, REF_CS_BGR = 3, REF_CS_GBR = 4, REF_CS_YCBCR = 16, REF_CS_BT601 = 17, REF_CS_SMPTE170M = 18,
       REF_CS_BT709 = 19, REF_CS_SMPTE240M = 20, REF_CS_BT2020 = 21 };

} // extern "C"

namespace {

bool csIsRGB(int32 c) { return c == REF_CS_RGB || c == REF_CS_BGR || c == REF_CS_GBR; }
bool csIsDefinedYCbCr(int32 c) { return c > REF_CS_YCBCR; }
eClrSpcLC csToLC(int32 c)
{
  switch(c)
  {
  case REF_CS_BT601: return eClrSpcLC::BT601;
  case REF_CS_SMPTE170M: return eClrSpcLC::SMPTE170M;
  case REF_CS_BT709: return eClrSpcLC::BT709;
  case REF_CS_SMPTE240M: return eClrSpcLC::SMPTE240M;
  case REF_CS_BT2020: return eClrSpcLC::BT2020;
  default: return eClrSpcLC::INVALID;
  }
}

// The colour part of xAppQMIV::preprocessFrames (apps/QMIV/src/xAppQMIV.cpp:856-891, flags from :302-311)
// on the two loaded 4:4:4 pictures.
void convertColour(xPicP* Pic, int32 CsIn, int32 CsMetric)
{
  const bool CvtYCbCr2RGB = csIsDefinedYCbCr(CsIn) && csIsRGB(CsMetric);
  const bool CvtRGB2YCbCr = csIsRGB(CsIn) && csIsDefinedYCbCr(CsMetric);
  const bool ReorderRGB   = csIsRGB(CsIn) && CsIn != REF_CS_RGB && CsMetric == REF_CS_RGB;
  for(int32 i = 0; i < 2; i++)
  {
    xPicP& P = Pic[i];
    if(CvtYCbCr2RGB)
    {
      xColorSpace::ConvertYCbCr2RGB(P.getAddr(eCmp::R), P.getAddr(eCmp::G), P.getAddr(eCmp::B), P.getAddr(eCmp::LM), P.getAddr(eCmp::CB),
                                    P.getAddr(eCmp::CR), P.getStride(), P.getStride(), P.getWidth(), P.getHeight(), P.getBitDepth(), csToLC(CsIn));
    }
    if(CvtRGB2YCbCr)
    {
      xColorSpace::ConvertRGB2YCbCr(P.getAddr(eCmp::LM), P.getAddr(eCmp::CB), P.getAddr(eCmp::CR), P.getAddr(eCmp::R), P.getAddr(eCmp::G),
                                    P.getAddr(eCmp::B), P.getStride(), P.getStride(), P.getWidth(), P.getHeight(), P.getBitDepth(), csToLC(CsMetric));
    }
    if(ReorderRGB)
    {
      if(CsIn == REF_CS_BGR) { P.swapComponents(eCmp::C0, eCmp::C2); }
      if(CsIn == REF_CS_GBR) { P.swapComponents(eCmp::C0, eCmp::C1); P.swapComponents(eCmp::C0, eCmp::C2); }
    }
  }
}

int computePairImpl(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3], uint32_t Mask, ref_result* Out,
                    uint16_t* Scp0, uint16_t* Scp1, int32 CsIn, int32 CsMetric, const ref_ssim_cfg* Ssim);

const ref_ssim_cfg c_DefaultSsim = { (int32_t)xSSIM::eMode::BlockAveraged, (int32_t)eMrgExt::None, 8, 4 };

} // namespace

extern "C" {

/* Full per-frame pipeline of the reference app for one frame pair. scp0/scp1 (optional, 3*W*H uint16
   each, planar) receive the shift-compensated pictures m_PicSCP[0] / m_PicSCP[1]. Returns 0 on success. */
int ref_compute_pair(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3], uint32_t Mask, ref_result* Out, uint16_t* Scp0, uint16_t* Scp1)
{
  return computePairImpl(P, Planes0, Planes1, Mask, Out, Scp0, Scp1, REF_CS_YCBCR, REF_CS_YCBCR, &c_DefaultSsim);
}

/* The same with the app's colour-space options: input colour space CsIn (-csi) and metric colour
   space CsMetric (-csm), codes as eClrSpcApp. */
int ref_compute_pair_cs(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3], uint32_t Mask, int32_t CsIn,
                        int32_t CsMetric, ref_result* Out)
{
  return computePairImpl(P, Planes0, Planes1, Mask, Out, nullptr, nullptr, CsIn, CsMetric, &c_DefaultSsim);
}

/* The same with the app's structural similarity options. With a border mode the pictures get a margin
   of at least 6 so that every 11x11 window read lands in the extended margin (the app's own margin is
   roundUp(R, 2), xAppQMIV.cpp:353, narrower than the 5-sample window reach for R <= 4). */
int ref_compute_pair_ssim(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3], uint32_t Mask,
                          const ref_ssim_cfg* Ssim, ref_result* Out)
{
  return computePairImpl(P, Planes0, Planes1, Mask, Out, nullptr, nullptr, REF_CS_YCBCR, REF_CS_YCBCR, Ssim);
}

} // extern "C"

namespace {

int computePairImpl(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3], uint32_t Mask, ref_result* Out,
                    uint16_t* Scp0, uint16_t* Scp1, int32 CsIn, int32 CsMetric, const ref_ssim_cfg* Ssim)
{
  const int32   W = P->width, H = P->height, BD = P->bitdepth;
  const int32V2 Size = { W, H };
  const eMrgExt Border = (eMrgExt)Ssim->border;
  const int32   Margin = xRoundUpToNearestMultiple(Border != eMrgExt::None ? xMax(P->search_range, 5) : P->search_range, 2);
  const int32V4 Cws = { P->cws[0], P->cws[1], P->cws[2], P->cws[3] };
  const int32V4 Cwa = { P->cwa[0], P->cwa[1], P->cwa[2], P->cwa[3] };
  const flt32V4 Unc = { P->unc[0], P->unc[1], P->unc[2], P->unc[3] };

  const bool CalcPSNRs = Mask & (REF_PSNR | REF_WSPSNR | REF_IVPSNR);
  const bool CalcSSIMs = Mask & (REF_SSIM | REF_MSSSIM | REF_IVSSIM | REF_IVMSSSIM);
  const bool CalcMSs   = Mask & (REF_MSSSIM | REF_IVMSSSIM);
  const bool CalcSCP   = (Mask & (REF_IVSSIM | REF_IVMSSSIM)) || Scp0 || Scp1;
  const bool CalcGCD   = (Mask & (REF_IVPSNR | REF_IVSSIM | REF_IVMSSSIM)) || CalcSCP;

  Pool TP(P->num_threads, H);

  xPicP PicP[2]; xPicI PicI[2]; xPicP SCP[2]; xPicI SCI[2];
  for(int32 i = 0; i < 2; i++) { PicP[i].create(Size, BD, Margin); PicI[i].create(Size, BD, Margin); }
  if(CalcSCP) { for(int32 i = 0; i < 2; i++) { SCP[i].create(Size, BD, Margin); SCI[i].create(Size, BD, Margin); } }

  loadFrame(PicP[0], Planes0, W, H, BD, P->chroma_format);
  loadFrame(PicP[1], Planes1, W, H, BD, P->chroma_format);
  convertColour(PicP, CsIn, CsMetric);

  std::memset(Out, 0, sizeof(ref_result));
  bool Exact[3];
  for(int32 c = 0; c < 3; c++) { Exact[c] = PicP[0].equalCmp(&PicP[1], (eCmp)c); Out->exact[c] = Exact[c]; }
  for(int32 i = 0; i < 2; i++) { PicP[i].extend(); }
  for(int32 i = 0; i < 2; i++) { PicI[i].rearrangeFromPlanar(&PicP[i]); }

  xGlobClrDiffProc ProcGCD; xShftCompPicProc ProcSCP; xIVPSNRM ProcPSNR; xIVSSIM ProcSSIM;
  ProcGCD.setUnntcbCoef(Unc); ProcGCD.bindThrdPoolIntf(&TP.TPI);
  ProcSCP.setSearchRange(P->search_range); ProcSCP.setCmpWeightsSearch(Cws); ProcSCP.setCmpWeightsAverage(Cwa); ProcSCP.bindThrdPoolIntf(&TP.TPI);
  if(CalcPSNRs)
  {
    ProcPSNR.setSearchRange(P->search_range); ProcPSNR.setCmpWeightsSearch(Cws); ProcPSNR.setCmpWeightsAverage(Cwa);
    ProcPSNR.setUnntcbCoef(Unc); ProcPSNR.bindThrdPoolIntf(&TP.TPI); ProcPSNR.initRowBuffers(H);
    if(P->erp) { ProcPSNR.initWS(true, W, H, BD, P->lon_range, P->lat_range); }
  }
  if(CalcSSIMs)
  {
    ProcSSIM.create(Size, BD, Margin, CalcMSs);
    ProcSSIM.setSearchRange(P->search_range); ProcSSIM.setCmpWeightsSearch(Cws); ProcSSIM.setCmpWeightsAverage(Cwa);
    ProcSSIM.setUnntcbCoef(Unc);
    ProcSSIM.setStructSimParams((xSSIM::eMode)Ssim->mode, Border, Ssim->window, Ssim->stride);
    ProcSSIM.bindThrdPoolIntf(&TP.TPI); ProcSSIM.initRowBuffers(H);
    if(P->erp) { ProcSSIM.initWS(true, W, H, BD, P->lon_range, P->lat_range); }
  }

  flt64 LastR2T = 0, LastT2R = 0;
  ProcPSNR.setDebugCallbackQAP([&](flt64 R2T, flt64 T2R) { LastR2T = R2T; LastT2R = T2R; });
  ProcSSIM.setDebugCallbackQAP([&](flt64 R2T, flt64 T2R) { LastR2T = R2T; LastT2R = T2R; });

  // per-picture average as xMetricStat::setPerCmpMeric (apps/QMIV/src/xMetricQMIV.cpp:91-97)
  const flt64 InvDen = 1.0 / (flt64)Cwa.getSum();
  auto PerPic = [&](const flt64V4& V) { return (V[0] * Cwa[0] + V[1] * Cwa[1] + V[2] * Cwa[2]) * InvDen; };

  int32V4 GCD = { 0, 0, 0, 0 };
  if(CalcGCD) { GCD = ProcGCD.CalcGlobalColorDiff(&PicP[0], &PicP[1]); }
  for(int32 c = 0; c < 4; c++) { Out->gcd_r2t[c] = GCD[c]; }

  if(CalcSCP)
  {
    ProcSCP.GenShftCompPics(&SCI[1], &SCI[0], &PicI[1], &PicI[0], GCD);
    for(int32 i = 0; i < 2; i++) { SCI[i].rearrangeToPlanar(&SCP[i]); }
    if(Scp0) { copyPlanar(Scp0, SCP[0], W, H); }
    if(Scp1) { copyPlanar(Scp1, SCP[1], W, H); }
  }

  if(Mask & REF_PSNR)
  {
    flt64V4 V = ProcPSNR.calcPicPSNR(&PicP[0], &PicP[1]);
    for(int32 c = 0; c < 3; c++) { if(Exact[c]) { V[c] = ProcPSNR.getFakePSNR(PicP[0].getArea(), PicP[0].getBitDepth()); } }
    for(int32 c = 0; c < 3; c++) { Out->psnr[c] = V[c]; }
    Out->psnr_pic = PerPic(V);
  }
  if(Mask & REF_WSPSNR)
  {
    flt64V4 V = ProcPSNR.calcPicWSPSNR(&PicP[0], &PicP[1]);
    for(int32 c = 0; c < 3; c++) { if(Exact[c]) { V[c] = ProcPSNR.getFakePSNR(PicP[0].getArea(), PicP[0].getBitDepth()); } }
    for(int32 c = 0; c < 3; c++) { Out->wspsnr[c] = V[c]; }
    Out->wspsnr_pic = PerPic(V);
  }
  if(Mask & REF_IVPSNR)
  {
    Out->ivpsnr = ProcPSNR.calcPicIVPSNR(&PicI[0], &PicI[1], GCD);
    Out->ivpsnr_r2t = LastR2T; Out->ivpsnr_t2r = LastT2R;
  }
  if(Border != eMrgExt::None)  // xAppQMIV::addStructSimMargs (xAppQMIV.cpp:798, 918-926)
  {
    for(int32 i = 0; i < 2; i++) { PicP[i].extend(Border); }
    if(CalcSCP) { for(int32 i = 0; i < 2; i++) { SCP[i].extend(Border); } }
  }
  if(Mask & REF_SSIM)
  {
    flt64V4 V = ProcSSIM.calcPicSSIM(&PicP[0], &PicP[1]);
    for(int32 c = 0; c < 3; c++) { Out->ssim[c] = V[c]; }
    Out->ssim_pic = PerPic(V);
  }
  if(Mask & REF_MSSSIM)
  {
    flt64V4 V = ProcSSIM.calcPicMSSSIM(&PicP[0], &PicP[1]);
    for(int32 c = 0; c < 3; c++) { Out->msssim[c] = V[c]; }
    Out->msssim_pic = PerPic(V);
  }
  if(Mask & REF_IVSSIM)
  {
    Out->ivssim = ProcSSIM.calcPicIVSSIM(&PicP[0], &PicP[1], &SCP[0], &SCP[1]);
    Out->ivssim_r2t = LastR2T; Out->ivssim_t2r = LastT2R;
  }
  if(Mask & REF_IVMSSSIM)
  {
    Out->ivmsssim = ProcSSIM.calcPicIVMSSSIM(&PicP[0], &PicP[1], &SCP[0], &SCP[1]);
    Out->ivmsssim_r2t = LastR2T; Out->ivmsssim_t2r = LastT2R;
  }

  if(CalcSSIMs) { ProcSSIM.destroy(); }
  return 0;
}

} // namespace

extern "C" {

/* Mask mode of the reference app for one frame pair: the mask picture's luma (W x H, 1 byte per
   sample for MaskBitDepth 8, else 2 bytes) weights every sample; metrics limited to PSNR, WS-PSNR and
   IV-PSNR as the app requires (xAppQMIV.cpp:360-365). NumNonMasked receives CountNonZero(mask). */
int ref_compute_pair_masked(const ref_params* P, const void* const Planes0[3], const void* const Planes1[3],
                            const void* MaskPlane, int32_t MaskBitDepth, uint32_t Mask, ref_result* Out, int32_t* NumNonMaskedOut)
{
  const int32   W = P->width, H = P->height, BD = P->bitdepth;
  const int32V2 Size = { W, H };
  const int32   Margin = xRoundUpToNearestMultiple(P->search_range, 2);
  const int32V4 Cws = { P->cws[0], P->cws[1], P->cws[2], P->cws[3] };
  const int32V4 Cwa = { P->cwa[0], P->cwa[1], P->cwa[2], P->cwa[3] };
  const flt32V4 Unc = { P->unc[0], P->unc[1], P->unc[2], P->unc[3] };
  if(Mask & (REF_SSIM | REF_MSSSIM | REF_IVSSIM | REF_IVMSSSIM)) { return 1; }

  Pool TP(P->num_threads, H);

  xPicP PicP[3]; xPicI PicI[2];
  for(int32 i = 0; i < 2; i++) { PicP[i].create(Size, BD, Margin); PicI[i].create(Size, BD, Margin); }
  PicP[2].create(Size, MaskBitDepth, Margin);
  loadFrame(PicP[0], Planes0, W, H, BD, P->chroma_format);
  loadFrame(PicP[1], Planes1, W, H, BD, P->chroma_format);
  // the mask file is read like the inputs; only its luma is used (eCmp::LM in every *M call)
  if(MaskBitDepth <= 8) { xPixelOps::Cvt(PicP[2].getAddr(eCmp::LM), (const uint8*)MaskPlane, PicP[2].getStride(), W, W, H); }
  else                  { xPixelOps::Copy(PicP[2].getAddr(eCmp::LM), (const uint16*)MaskPlane, PicP[2].getStride(), W, W, H); }
  for(int32 c = 1; c < 3; c++) { PicP[2].fill(0, (eCmp)c); }

  std::memset(Out, 0, sizeof(ref_result));
  bool Exact[3];
  for(int32 c = 0; c < 3; c++) { Exact[c] = PicP[0].equalCmp(&PicP[1], (eCmp)c); Out->exact[c] = Exact[c]; }
  for(int32 i = 0; i < 3; i++) { PicP[i].extend(); }
  const int32 NumNonMasked = xPixelOps::CountNonZero(PicP[2].getAddr(eCmp::LM), PicP[2].getStride(), W, H);
  *NumNonMaskedOut = NumNonMasked;
  for(int32 i = 0; i < 2; i++) { PicI[i].rearrangeFromPlanar(&PicP[i]); }

  xGlobClrDiffProc ProcGCD; xIVPSNRM ProcPSNR;
  ProcGCD.setUnntcbCoef(Unc); ProcGCD.bindThrdPoolIntf(&TP.TPI);
  ProcPSNR.setSearchRange(P->search_range); ProcPSNR.setCmpWeightsSearch(Cws); ProcPSNR.setCmpWeightsAverage(Cwa);
  ProcPSNR.setUnntcbCoef(Unc); ProcPSNR.bindThrdPoolIntf(&TP.TPI); ProcPSNR.initRowBuffers(H);
  if(P->erp) { ProcPSNR.initWS(true, W, H, BD, P->lon_range, P->lat_range); }

  flt64 LastR2T = 0, LastT2R = 0;
  ProcPSNR.setDebugCallbackQAP([&](flt64 R2T, flt64 T2R) { LastR2T = R2T; LastT2R = T2R; });
  const flt64 InvDen = 1.0 / (flt64)Cwa.getSum();
  auto PerPic = [&](const flt64V4& V) { return (V[0] * Cwa[0] + V[1] * Cwa[1] + V[2] * Cwa[2]) * InvDen; };

  int32V4 GCD = { 0, 0, 0, 0 };
  if(Mask & REF_IVPSNR) { GCD = ProcGCD.CalcGlobalColorDiffM(&PicP[0], &PicP[1], &PicP[2], NumNonMasked); }
  for(int32 c = 0; c < 4; c++) { Out->gcd_r2t[c] = GCD[c]; }

  if(Mask & REF_PSNR)
  {
    flt64V4 V = ProcPSNR.calcPicPSNRM(&PicP[0], &PicP[1], &PicP[2], NumNonMasked);
    for(int32 c = 0; c < 3; c++) { if(Exact[c]) { V[c] = ProcPSNR.getFakePSNR(PicP[0].getArea(), PicP[0].getBitDepth()); } }
    for(int32 c = 0; c < 3; c++) { Out->psnr[c] = V[c]; }
    Out->psnr_pic = PerPic(V);
  }
  if(Mask & REF_WSPSNR)
  {
    flt64V4 V = ProcPSNR.calcPicWSPSNRM(&PicP[0], &PicP[1], &PicP[2], NumNonMasked);
    for(int32 c = 0; c < 3; c++) { if(Exact[c]) { V[c] = ProcPSNR.getFakePSNR(PicP[0].getArea(), PicP[0].getBitDepth()); } }
    for(int32 c = 0; c < 3; c++) { Out->wspsnr[c] = V[c]; }
    Out->wspsnr_pic = PerPic(V);
  }
  if(Mask & REF_IVPSNR)
  {
    Out->ivpsnr = ProcPSNR.calcPicIVPSNRM(&PicI[0], &PicI[1], &PicP[2], NumNonMasked, GCD);
    Out->ivpsnr_r2t = LastR2T; Out->ivpsnr_t2r = LastT2R;
  }
  return 0;
}

/* Per-row CPS distortion of one direction on 4:4:4 planar uint16 pictures (3*W*H each), through both the
   x86 interleaved path (xCorrespPixelShiftSSE, what the app dispatches to) and the portable planar path
   (xCorrespPixelShiftSTD). row_sse_* receive H*3 uint64 values. Margin = roundUp(R,2) filled by extend(). */
int ref_cps_rows(const uint16_t* Tst, const uint16_t* Ref, int32_t W, int32_t H, int32_t BitDepth, const int32_t Gcd[4], int32_t R, const int32_t Cws[4], uint64_t* RowSseInterleaved, uint64_t* RowSsePlanar)
{
  const int32V2 Size   = { W, H };
  const int32   Margin = xRoundUpToNearestMultiple(R, 2);
  xPicP TP(Size, BitDepth, Margin), RP(Size, BitDepth, Margin);
  for(int32 c = 0; c < 3; c++)
  {
    xPixelOps::Copy(TP.getAddr((eCmp)c), Tst + (size_t)c * W * H, TP.getStride(), W, W, H);
    xPixelOps::Copy(RP.getAddr((eCmp)c), Ref + (size_t)c * W * H, RP.getStride(), W, W, H);
  }
  TP.extend(); RP.extend();
  xPicI TI(Size, BitDepth, Margin), RI(Size, BitDepth, Margin);
  TI.rearrangeFromPlanar(&TP); RI.rearrangeFromPlanar(&RP);
  const int32V4 G = { Gcd[0], Gcd[1], Gcd[2], Gcd[3] };
  const int32V4 Wt = { Cws[0], Cws[1], Cws[2], Cws[3] };
  for(int32 y = 0; y < H; y++)
  {
    uint64V4 A = xCorrespPixelShift::CalcDistAsymmetricRow(&TI, &RI, y, G, R, Wt);
    uint64V4 B = xCorrespPixelShift::CalcDistAsymmetricRow(&TP, &RP, y, G, R, Wt);
    for(int32 c = 0; c < 3; c++) { RowSseInterleaved[y * 3 + c] = A[c]; RowSsePlanar[y * 3 + c] = B[c]; }
  }
  return 0;
}

/* Raw xGlobClrDiff::CalcGlobalColorDiff(Tst, Ref, coef) on 4:4:4 planar uint16 pictures. */
int ref_gcd(const uint16_t* Tst, const uint16_t* Ref, int32_t W, int32_t H, int32_t BitDepth, const float Coef[4], int32_t Out[4])
{
  const int32V2 Size = { W, H };
  xPicP TP(Size, BitDepth, 0), RP(Size, BitDepth, 0);
  for(int32 c = 0; c < 3; c++)
  {
    xPixelOps::Copy(TP.getAddr((eCmp)c), Tst + (size_t)c * W * H, TP.getStride(), W, W, H);
    xPixelOps::Copy(RP.getAddr((eCmp)c), Ref + (size_t)c * W * H, RP.getStride(), W, W, H);
  }
  int32V4 G = xGlobClrDiff::CalcGlobalColorDiff(&TP, &RP, { Coef[0], Coef[1], Coef[2], Coef[3] }, nullptr);
  for(int32 c = 0; c < 4; c++) { Out[c] = G[c]; }
  return 0;
}

/* Block-averaged SSIM of one 8x8 window (xStructSim::CalcBlckAvg dispatch and the portable STD version). */
double ref_ssim_block(const uint16_t* Tst, const uint16_t* Ref, int32_t StrideT, int32_t StrideR, int32_t BitDepth, int32_t CalcL, int32_t UseStd)
{
  const flt64 MaxValue = (flt64)xBitDepth2MaxValue(BitDepth);
  const flt64 C1 = xPow2(xStructSimConsts::c_K1<flt64> * MaxValue);
  const flt64 C2 = xPow2(xStructSimConsts::c_K2<flt64> * MaxValue);
  if(UseStd) { return xStructSimSTD::CalcBlckAvg(Tst, Ref, StrideT, StrideR, 8, C1, C2, CalcL != 0); }
  return xStructSim::CalcBlckAvg(Tst, Ref, StrideT, StrideR, 8, C1, C2, CalcL != 0);
}

/* Test-fixture generators of the reference's unit tests (xTestUtils.h, xTestUtilsIVQM.cpp). */
uint32_t ref_xorshift32(uint32_t State) { return xTestUtils::xXorShift32(State); }
void ref_fill_perlin(uint16_t* Dst, int32_t Stride, int32_t W, int32_t H, int32_t BitDepth, int32_t Octaves, uint32_t Seed)
{
  xPerlinNoise::fillPerlinNoiseI(Dst, Stride, W, H, BitDepth, Octaves, Seed);
}
uint32_t ref_add_block_noise(uint16_t* Dst, const uint16_t* Src, int32_t DstStride, int32_t SrcStride, int32_t W, int32_t H, int32_t BitDepth, uint32_t State)
{
  return xTestUtilsIVQM::addBlockNoise(Dst, Src, DstStride, SrcStride, W, H, BitDepth, State);
}

} // extern "C"
