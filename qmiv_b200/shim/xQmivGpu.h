// Drop-in adapter for a QMIV host: the app's per-frame metric calls on its own pictures
// (apps/QMIV/src/xAppQMIV.cpp:927-1108, processors set up at :680-744) become one call per frame pair
// into this library's C ABI (include/qmiv_gpu.h).
//
// The host keeps its pictures as the reference reads them: xPicP (libs/pmbb-core/src/xPic.h:19),
// planar uint16 4:4:4 (chroma already upsampled by xSeqPic::xUnpackFrame) with a margin around the
// picture, addressed from the origin of each component with the picture's stride. calcFrame() hands
// those planes, in place, to a 4:4:4 calc of the same size and bit depth; the library uploads them
// and runs the whole metric pipeline on the GPU. Pictures of 8 bits or less are packed to one byte
// per sample first (the library's sample size follows the bit depth), into buffers the adapter keeps.
// Metrics computed on the 4:4:4 pictures equal the reference's on the same pictures, which is what
// the reference computes from 4:2:0 input too (it upsamples before every metric).
//
// Build: compile xQmivGpu.cpp with the host's pmbb include directories and PMBB_NAMESPACE defined as
// the host defines it, add this repository's include/ directory, link libqmiv_b200.so.
#pragma once

#include "xPic.h"
#include "qmiv_gpu.h"

#include <vector>

namespace PMBB_NAMESPACE {

class xQmivGpu
{
protected:
  qmiv_ctx  m_Ctx      = nullptr;
  qmiv_calc m_Calc     = nullptr;
  int32V2   m_Size     = { 0, 0 };
  int32     m_BitDepth = 0;
  std::vector<uint8> m_Packed[2];   // byte planes of the last frame pair (bit depth <= 8)

public:
  xQmivGpu() = default;
  xQmivGpu(const xQmivGpu&) = delete;
  xQmivGpu& operator=(const xQmivGpu&) = delete;
  ~xQmivGpu() { destroy(); }

  // Device: CUDA ordinal. Params: the processors' settings (search range, search and average weights,
  // unnoticeable coefficients, ERP ranges, structural similarity options; NULL = the app's defaults).
  qmiv_status create (int32 Device, int32V2 Size, int32 BitDepth, const qmiv_params* Params = nullptr);
  void        destroy();
  bool        isCreated() const { return m_Calc != nullptr; }

  // Every metric in MetricMask (QMIV_PSNR, QMIV_WSPSNR, QMIV_IVPSNR, QMIV_SSIM, QMIV_MSSSIM,
  // QMIV_IVSSIM, QMIV_IVMSSSIM) of the pair (Pic0 = In0, Pic1 = In1), in one pass on the GPU. The
  // pictures must match the size and bit depth given to create(); their margins are not read.
  qmiv_status calcFrame(const xPicP* Pic0, const xPicP* Pic1, uint32 MetricMask, qmiv_result* Result);

  // One metric per call, in the value types of the reference's processors (xPSNR::calcPicPSNR,
  // xWSPSNR::calcPicWSPSNR, xIVPSNR::calcPicIVPSNR, xSSIM::calcPicSSIM / calcPicMSSSIM,
  // xIVSSIM::calcPicIVSSIM / calcPicIVMSSSIM); NaN where the call fails. A host that needs several
  // metrics of one pair calls calcFrame() once instead.
  flt64V4 calcPicPSNR    (const xPicP* Pic0, const xPicP* Pic1);
  flt64V4 calcPicWSPSNR  (const xPicP* Pic0, const xPicP* Pic1);
  flt64   calcPicIVPSNR  (const xPicP* Pic0, const xPicP* Pic1);
  flt64V4 calcPicSSIM    (const xPicP* Pic0, const xPicP* Pic1);
  flt64V4 calcPicMSSSIM  (const xPicP* Pic0, const xPicP* Pic1);
  flt64   calcPicIVSSIM  (const xPicP* Pic0, const xPicP* Pic1);
  flt64   calcPicIVMSSSIM(const xPicP* Pic0, const xPicP* Pic1);

protected:
  qmiv_status xBindFrame(const xPicP* Pic, int32 Slot, qmiv_frame* Frame);
};

} // end of namespace PMBB_NAMESPACE
