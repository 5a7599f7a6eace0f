// TEST INFRASTRUCTURE ONLY: checks the drop-in adapter qmiv_b200/shim/xQmivGpu.cpp on the reference's
// own picture type. Built by oracle/Makefile (target shimcheck) from the reference's library objects,
// the adapter and libqmiv_b200.so.
//
//   shim_check W H bitdepth chroma_format search_range erp metric_mask frame0.yuv frame1.yuv
//
// Reads two raw planar frames, fills 4:4:4 xPicP pictures (libs/pmbb-core/src/xPic.h:19) the way the
// reference's loader does (nearest chroma upsampling, libs/pmbb-core/src/xSeq.cpp:231-290), runs
// xQmivGpu::calcFrame with the given metrics and the single-metric calls of the adapter, and prints
// every value as JSON with doubles in hexadecimal (exact).
#include "xQmivGpu.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace PMBB_NAMESPACE;

static bool readFrame(const char* Path, int32 W, int32 H, int32 BitDepth, int32 ChromaFormat, xPicP& Pic)
{
  const int32 sx = ChromaFormat == 444 ? 0 : 1, sy = ChromaFormat == 420 ? 1 : 0;
  const int32 cw = W >> sx, ch = H >> sy, bytes = BitDepth <= 8 ? 1 : 2;
  const size_t n = (size_t)W * H + 2 * (size_t)cw * ch;
  std::vector<uint8> raw(n * bytes);
  FILE* f = std::fopen(Path, "rb");
  if(!f) { return false; }
  const size_t got = std::fread(raw.data(), 1, raw.size(), f);
  std::fclose(f);
  if(got != raw.size()) { return false; }
  auto sample = [&](size_t i) -> uint16 { return bytes == 1 ? raw[i] : (uint16)(raw[2 * i] | (raw[2 * i + 1] << 8)); };
  const size_t off[3] = { 0, (size_t)W * H, (size_t)W * H + (size_t)cw * ch };
  for(int32 c = 0; c < 3; c++)
  {
    uint16* Dst = Pic.getAddr((eCmp)c);
    const int32 psx = c ? sx : 0, psy = c ? sy : 0, pw = c ? cw : W;
    for(int32 y = 0; y < H; y++)
    {
      for(int32 x = 0; x < W; x++) { Dst[(size_t)y * Pic.getStride() + x] = sample(off[c] + (size_t)(y >> psy) * pw + (x >> psx)); }
    }
  }
  Pic.extend();   // the app extends its pictures before the metrics; the adapter does not read margins
  return true;
}

static void put(const char* Key, double V, bool Last = false) { std::printf("\"%s\": \"%a\"%s", Key, V, Last ? "" : ", "); }
static void put4(const char* Key, const double* V)
{
  std::printf("\"%s\": [\"%a\", \"%a\", \"%a\"], ", Key, V[0], V[1], V[2]);
}

int main(int argc, char** argv)
{
  if(argc != 10) { std::fprintf(stderr, "usage: shim_check W H bitdepth chroma_format R erp mask frame0 frame1\n"); return 2; }
  const int32 W = std::atoi(argv[1]), H = std::atoi(argv[2]), BD = std::atoi(argv[3]), CF = std::atoi(argv[4]);
  const int32 R = std::atoi(argv[5]), Erp = std::atoi(argv[6]);
  const uint32 Mask = (uint32)std::strtoul(argv[7], nullptr, 0);
  xPicP Pic[2];
  for(int32 i = 0; i < 2; i++)
  {
    Pic[i].create(int32V2(W, H), BD, 8);
    if(!readFrame(argv[8 + i], W, H, BD, CF, Pic[i])) { std::fprintf(stderr, "cannot read %s\n", argv[8 + i]); return 2; }
  }
  qmiv_params Prm;
  qmiv_params_default(&Prm);
  Prm.search_range = R;
  Prm.erp = Erp;
  xQmivGpu Gpu;
  qmiv_status s = Gpu.create(0, int32V2(W, H), BD, &Prm);
  if(s != QMIV_OK) { std::fprintf(stderr, "create: %s\n", qmiv_last_error()); return 1; }
  qmiv_result Res{};
  s = Gpu.calcFrame(&Pic[0], &Pic[1], Mask, &Res);
  if(s != QMIV_OK) { std::fprintf(stderr, "calcFrame: %s\n", qmiv_last_error()); return 1; }
  std::printf("{");
  std::printf("\"gcd_r2t\": [%d, %d, %d], ", Res.gcd_r2t[0], Res.gcd_r2t[1], Res.gcd_r2t[2]);
  put4("psnr", Res.psnr); put("psnr_pic", Res.psnr_pic);
  put4("wspsnr", Res.wspsnr); put("wspsnr_pic", Res.wspsnr_pic);
  put("ivpsnr", Res.ivpsnr); put("ivpsnr_r2t", Res.ivpsnr_r2t); put("ivpsnr_t2r", Res.ivpsnr_t2r);
  put4("ssim", Res.ssim); put("ssim_pic", Res.ssim_pic);
  put4("msssim", Res.msssim); put("msssim_pic", Res.msssim_pic);
  put("ivssim", Res.ivssim); put("ivssim_r2t", Res.ivssim_r2t); put("ivssim_t2r", Res.ivssim_t2r);
  put("ivmsssim", Res.ivmsssim); put("ivmsssim_r2t", Res.ivmsssim_r2t); put("ivmsssim_t2r", Res.ivmsssim_t2r);
  // the single-metric calls of the adapter on the same pictures
  const flt64V4 P = Gpu.calcPicPSNR(&Pic[0], &Pic[1]);
  const flt64V4 S = Gpu.calcPicSSIM(&Pic[0], &Pic[1]);
  put("one_psnr_y", P[0]); put("one_ivpsnr", Gpu.calcPicIVPSNR(&Pic[0], &Pic[1])); put("one_ssim_y", S[0]);
  put("one_ivssim", Gpu.calcPicIVSSIM(&Pic[0], &Pic[1]), true);
  std::printf("}\n");
  return 0;
}
