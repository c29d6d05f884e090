// Known-answer and error-path checks of the header-only C++ driver layer
// (include/ctstereo.hpp), written the way a reference user drives
// Clu::Cuda::*::CDriver: Configure -> ProcessKernel -> CopyInto.
//
//   shim_test cpu               argument checks that never reach a device
//   shim_test gpu <weights.f32> every driver on a pair whose right image is
//                               the left one shifted by a known disparity
//
// Exit status 0 = all checks passed; each failure prints one line.
#include "ctstereo.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <random>
#include <string>
#include <vector>

using namespace ctstereo;

static int g_failures = 0;

#define CHECK(cond, ...)                                  \
    do {                                                  \
        if (!(cond)) {                                    \
            std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
            std::printf(__VA_ARGS__);                     \
            std::printf("\n");                            \
            ++g_failures;                                 \
        }                                                 \
    } while (0)

// Runs f and returns the CError code it threw (0 if none, -1 for another exception).
static int ThrownCode(const std::function<void()>& f) {
    try {
        f();
    } catch (const CError& e) {
        if (std::strlen(e.what()) == 0) return -2;
        return e.Code();
    } catch (...) {
        return -1;
    }
    return 0;
}

static int RunCpu() {
    const CDevice dev(0);
    const SImageFormat f(320, 120);

    BlockMatcherSAD1::SParameter sad;
    sad.Set(0, 64, 0, 0.f, 0.f, BlockMatcherSAD1::EConfig::Patch_9x9);
    CHECK(sad.iDispRange == 64 && sad.eConfig == BlockMatcherSAD1::EConfig::Patch_9x9, "SAD Set");
    {
        BlockMatcherSAD1::SParameter p = sad;
        BlockMatcherSAD1::CDriver d;
        p.iOffset = -1;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "SAD negative offset must be rejected");
        CHECK(ThrownCode([&] { d.Configure(dev, SImageFormat(320, 120, EDataType::UInt16), sad); }) == CT_ETYPE,
              "SAD UInt16 input must be rejected");
        p = sad;
        p.iDispRange = 0;  // reaches the C ABI, which checks before touching a device
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "SAD disp range 0 must be rejected");
    }
    {
        _SDisparityConfig dc;
        dc.Set(0, 128);
        BlockMatcherNCC::SParameter p;
        p.Set(dc, 0, 0.f, 0.f, 1, true, BlockMatcherNCC::EConfig::Patch_11x11);
        BlockMatcherNCC::CDriver d;
        CHECK(ThrownCode([&] { d.SetTensorCores(false); }) == CT_ESTATE, "NCC SetTensorCores before Configure");
        p.iUseDispInput = 0;
        p.xDispConfig.Set(-1, 128);
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "NCC iMin < 0 must be rejected");
        p.xDispConfig.Set(0, 300);
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "NCC range 300 must be rejected");
    }
    {
        _SDisparityConfig dc;
        dc.Set(0, 256);
        BlockMatcherAW1::SParameter p;
        p.Set(dc, 0.f, 0.f, 0.f, 1, true, BlockMatcherAW1::EConfig::Patch_15x15,
              BlockMatcherAW1::ESimType::AbsoluteDifference);
        BlockMatcherAW1::CDriver d;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "AW1 2-of-4 guided must be rejected");
        p.iUseDispInput = 0;
        p.eConfig = BlockMatcherAW1::EConfig::Shifted5_7x7;
        p.eSimType = BlockMatcherAW1::ESimType::SignedProduct;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "Shifted5_7x7 signed product must be rejected");
        p.eSimType = BlockMatcherAW1::ESimType::AbsoluteDifference;
        p.fSimThresh = 50.f;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "Shifted5_7x7 fSimThresh must be rejected");
    }
    {
        BlockMatcherAW2::SParameter p;
        p.Set(-2, 64, 0, 30.f, 0.f, 0, BlockMatcherAW2::EConfig::Patch_9x9);
        BlockMatcherAW2::CDriver d;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "AW2 negative offset must be rejected");
        p.Set(0, 64, 0, 30.f, 0.f, 1, BlockMatcherAW2::EConfig::Patch_9x9);
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "AW2 guided mode must be rejected");
    }
    {
        _SDisparityConfig dc;
        dc.Set(0, 64);
        BlockMatcher1::SParameter p;
        p.Set(dc, 0.f, 40.f, 0.f, 1, true, BlockMatcher1::EConfig::Patch_9x9, BlockMatcher1::ESimType::SignedProduct);
        BlockMatcher1::CDriver d;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "BM1 guided mode must be rejected");
        p.iUseDispInput = 0;
        p.xDispConfig.Set(0, 0);
        CHECK(ThrownCode([&] { d.Configure(dev, f, p); }) == CT_EINVAL, "BM1 range 0 must be rejected");
    }
    {
        CrossCheckDisparityMaps::SParameter p;
        _SDisparityConfig dc;
        dc.Set(0, 64);
        p.Set(dc, 1, 1);
        CrossCheckDisparityMaps::CDriver d;
        CHECK(ThrownCode([&] { d.Configure(dev, SImageFormat(320, 120, EDataType::UInt64), p); }) == CT_ETYPE,
              "cross-check on UInt64 maps must be rejected");
        p.iDispDeltaThresh = -1;
        CHECK(ThrownCode([&] { d.Configure(dev, SImageFormat(320, 120, EDataType::UInt16), p); }) == CT_EINVAL,
              "negative tolerance must be rejected");
    }
    {
        BatchStereo::CDriver d;
        CHECK(ThrownCode([&] { d.Configure(dev, {f, f}, {64}, 1); }) == CT_EINVAL, "batch shape/range mismatch");
    }
    {
        ConfidenceNet::CDriver d;
        CHECK(ThrownCode([&] { d.LoadParams("/nonexistent/weights.f32"); }) == CT_EINVAL, "missing weight file");
    }
    {
        CensusStream::CDriver d;
        BlockMatcherCensus::SParameter p;
        p.xDispConfig.Set(0, 64);
        p.bLeftToRight = false;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p, 1); }) == CT_EINVAL, "stream of right-view maps");
        p.bLeftToRight = true;
        CHECK(ThrownCode([&] { d.Configure(dev, f, p, 1, EDataType::Single); }) == CT_ETYPE, "F32 stream maps");
        CHECK(ThrownCode([&] { d.Submit(nullptr, 0, nullptr, 0, nullptr, 0); }) == CT_ESTATE, "unconfigured stream");
    }
    {
        // disparity to 3D: parameter checks before any device call
        MapDisparityTo3D::CStereoPinhole cams{};
        for (int c = 0; c < 2; ++c) cams.cam[c] = ct_pinhole{500.f, 500.f, 160.f, 60.f, {1, 0, 0, 0, 1, 0, 0, 0, 1}, {0.1f * c, 0, 0}};
        MapDisparityTo3D::SParameter mp;
        mp.Set(uint16_t(EDisparityId::First), uint16_t(EDisparityId::Last), true, cams);
        MapDisparityTo3D::CDriver m3;
        CHECK(ThrownCode([&] { m3.Configure(dev, SImageFormat(320, 120, EDataType::RGBA8), mp); }) == CT_ETYPE,
              "3D: RGBA8 disparity maps must be rejected");
        mp.camStereoPinhole.cam[1].fx = 0.f;
        CHECK(ThrownCode([&] { m3.Configure(dev, SImageFormat(320, 120, EDataType::UInt16), mp); }) == CT_EINVAL,
              "3D: a zero focal length must be rejected");
        mp.Set(90, 20, true, cams);
        CHECK(ThrownCode([&] { m3.Configure(dev, SImageFormat(320, 120, EDataType::UInt16), mp); }) == CT_EINVAL,
              "3D: disp_min above disp_max must be rejected");
        // mip-maps: the packed layout needs no device
        int32_t pw = 0, levels = 0;
        Ensure(ct_disp_mipmap_format(320, 120, &pw, &levels), "format");
        CHECK(pw == 320 + 159 && levels == 5, "mip-map format %d / %d", pw, levels);
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    if (n == 0) {
        // a valid configuration reaches the device and fails as a CUDA error
        BlockMatcherSAD1::CDriver d;
        const int code = ThrownCode([&] { d.Configure(dev, f, sad); });
        CHECK(code == CT_ECUDA, "configure without a device: code %d", code);
    }
    return g_failures;
}

// ---------------------------------------------------------------------------

static uint64_t HostCensus9x7(const std::vector<uint8_t>& img, int W, int x, int y) {
    uint64_t c = 0;
    const uint8_t ctr = img[size_t(y) * W + x];
    for (int dy = -3; dy <= 3; ++dy)
        for (int dx = -4; dx <= 4; ++dx) c = (c << 1) | uint64_t(img[size_t(y + dy) * W + x + dx] > ctr);
    return c;
}

static int RunGpu(const char* weights) {
    const int W = 320, H = 120, K = 7;  // right image = left shifted by K: L(x) = R(x - K)
    std::mt19937 rng(12345);
    std::vector<uint8_t> L(size_t(W) * H), R(size_t(W) * H);
    for (auto& v : L) v = uint8_t(rng() & 0xFF);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) R[size_t(y) * W + x] = x + K < W ? L[size_t(y) * W + x + K] : uint8_t(rng() & 0xFF);

    const CDevice dev(0);
    const SImageFormat fin(W, H);
    CDeviceSurface surfL(fin), surfR(fin);
    surfL.CopyFrom(L.data());
    surfR.CopyFrom(R.data());
    const SImageFormat f16(W, H, EDataType::UInt16), f8(W, H, EDataType::UInt8), f32(W, H, EDataType::Single);
    auto interior = [&](int x, int y, int r) { return y >= r && y < H - r && x >= K + r && x < W - r - K; };

    {  // census transform
        CensusTransform::CDriver d;
        d.Configure(dev, fin);
        CDeviceSurface desc(SImageFormat(W, H, EDataType::UInt64));
        const double ms = ProcessKernel(d, desc, surfL);
        CHECK(ms >= 0.0, "census time");
        auto got = desc.CopyInto<uint64_t>();
        int bad = 0;
        for (int y = 3; y < H - 3; ++y)
            for (int x = 4; x < W - 4; ++x) bad += got[size_t(y) * W + x] != HostCensus9x7(L, W, x, y);
        CHECK(bad == 0, "census: %d descriptors differ", bad);
    }
    {  // SAD 9x9, UInt8
        BlockMatcherSAD1::SParameter p;
        p.Set(0, 64, 0, 0.f, 0.f, BlockMatcherSAD1::EConfig::Patch_9x9);
        BlockMatcherSAD1::CDriver d;
        d.Configure(dev, fin, p);
        CDeviceSurface disp(f8);
        ProcessKernel(d, disp, surfL, surfR);
        auto v = disp.CopyInto<uint8_t>();
        int bad = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) bad += interior(x, y, 4) && v[size_t(y) * W + x] != K;
        CHECK(bad == 0, "SAD: %d interior pixels not at d = %d", bad, K);
    }
    {  // reference 4 x uint16 output of every driver on the shift: x = K + First
        const SImageFormat f4(W, H, EDataType::UInt16x4);
        auto check4 = [&](const char* who, CKernelDriverBase& drv, const std::function<void(CDeviceSurface&)>& run,
                          int r) {
            CDeviceSurface out(f4);
            drv.Begin();
            run(out);
            drv.End();
            auto v = out.CopyInto<uint64_t>();
            int bad = 0;
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x)
                    bad += interior(x, y, r + 1) && (v[size_t(y) * W + x] & 0xFFFF) != uint64_t(K + 1);
            CHECK(bad == 0, "%s (UInt16x4): %d interior pixels not at d = %d", who, bad, K);
        };
        BlockMatcherSAD1::SParameter ps;
        ps.Set(0, 32, 0, 1000.f, 0.f, BlockMatcherSAD1::EConfig::Patch_16x16);  // the reference's only patch
        BlockMatcherSAD1::CDriver sad;
        sad.Configure(dev, fin, ps);
        // (margin 12: at the left edge of the search the first evaluated
        // disparity can be the winner, whose "before" channel then reads the
        // scan's initial 0 and the pixel is NotSpecific, as in the reference)
        check4("SAD1 16x16", sad, [&](CDeviceSurface& o) { sad.Process(o, surfL, surfR); }, 12);
        CDeviceSurface plain(f16);  // Patch_16x16 has no plain map
        CHECK(ThrownCode([&] { sad.Process(plain, surfL, surfR); }) == CT_EINVAL, "SAD1 16x16 into UInt16");
        _SDisparityConfig dc;
        dc.Set(0, 32);
        BlockMatcherNCC::SParameter pn;
        pn.Set(dc, 0, 0.5f, 0.f, 0, true, BlockMatcherNCC::EConfig::Patch_11x11);
        BlockMatcherNCC::CDriver ncc;
        ncc.Configure(dev, fin, pn);
        check4("NCC", ncc, [&](CDeviceSurface& o) { ncc.Process(o, surfL, surfR); }, 5);
        CHECK(ThrownCode([&] { ncc.Process(plain, surfL, surfR); }) == CT_EINVAL,
              "fNccThresh on the plain map must be rejected");
        BlockMatcherAW1::SParameter pa;
        pa.Set(dc, 0.f, 50.f, 0.f, 0, true, BlockMatcherAW1::EConfig::Patch_15x15,
               BlockMatcherAW1::ESimType::AbsoluteDifference);
        BlockMatcherAW1::CDriver aw1;
        aw1.Configure(dev, fin, pa);
        check4("AW1 15x15", aw1, [&](CDeviceSurface& o) { aw1.Process(o, surfL, surfR); }, 7);
        BlockMatcherAW2::SParameter p2;
        p2.Set(0, 32, 0, 1000.f, 0.f, 0, BlockMatcherAW2::EConfig::Patch_9x9);
        BlockMatcherAW2::CDriver aw2;
        aw2.Configure(dev, fin, p2);
        check4("AW2 9x9", aw2, [&](CDeviceSurface& o) { aw2.Process(o, surfL, surfR); }, 4);
        BlockMatcher1::SParameter p1;
        p1.Set(dc, 0.f, 10.f, 0.f, 0, true, BlockMatcher1::EConfig::Patch_9x9, BlockMatcher1::ESimType::SignedProduct);
        BlockMatcher1::CDriver bm1;
        bm1.Configure(dev, fin, p1);
        check4("BM1 9x9", bm1, [&](CDeviceSurface& o) { bm1.Process(o, surfL, surfR); }, 4);
    }
    {  // NCC 11x11, UInt16 + score
        _SDisparityConfig dc;
        dc.Set(0, 128);
        BlockMatcherNCC::SParameter p;
        p.Set(dc, 0, 0.f, 0.f, 0, true, BlockMatcherNCC::EConfig::Patch_11x11);
        BlockMatcherNCC::CDriver d;
        d.Configure(dev, fin, p);
        CDeviceSurface disp(f16), score(f32);
        ProcessKernel(d, disp, surfL, surfR, _CDeviceSurface(), score);
        auto v = disp.CopyInto<uint16_t>();
        auto s = score.CopyInto<float>();
        int bad = 0, low = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                if (interior(x, y, 5)) {
                    bad += v[size_t(y) * W + x] != K + uint16_t(EDisparityId::First);
                    low += s[size_t(y) * W + x] < 0.9999f;
                }
        CHECK(bad == 0 && low == 0, "NCC: %d interior pixels off, %d scores below 1", bad, low);
        {  // the same map and scores with the window sums on the CUDA cores
            d.SetTensorCores(false);
            CDeviceSurface disp2(f16), score2(f32);
            ProcessKernel(d, disp2, surfL, surfR, _CDeviceSurface(), score2);
            d.SetTensorCores(true);
            const auto v2 = disp2.CopyInto<uint16_t>();
            const auto s2 = score2.CopyInto<float>();
            CHECK(v2 == v && std::memcmp(s2.data(), s.data(), s.size() * sizeof(float)) == 0,
                  "NCC: CUDA-core and tensor-core kernels differ");
        }

        // visualisation of the map: interior pixels gray at t = K / 128,
        // border pixels (CannotEvaluate) in the default colour
        ColorDisparityImage::SParameter cp;
        cp.Set(1, 129, 0);
        ColorDisparityImage::CDriver col;
        col.Configure(dev, f16, cp);
        CDeviceSurface rgba(SImageFormat(W, H, EDataType::RGBA8));
        ProcessKernel(col, rgba, disp, ColorDisparityImage::EStyle::Analysis);
        auto cv = rgba.CopyInto<uint32_t>();
        const uint32_t gray = uint32_t(std::lrint(float(K) / 128.f * 255.f));
        const uint32_t want_gray = gray | (gray << 8) | (gray << 16) | 0xFF000000u;
        CHECK(cv[size_t(60) * W + 100] == want_gray, "colour: interior %08x, want %08x", cv[size_t(60) * W + 100],
              want_gray);
        CHECK(cv[0] == cp.pixCannotEvaluate, "colour: border %08x, want %08x", cv[0], cp.pixCannotEvaluate);

        // 3D points of the map with a rectified pair (f = 500 px, baseline 0.2):
        // interior depth f B / K
        MapDisparityTo3D::CStereoPinhole cams{};
        for (int c = 0; c < 2; ++c) {
            cams.cam[c] = ct_pinhole{500.f, 500.f, W / 2.f, H / 2.f, {1, 0, 0, 0, 1, 0, 0, 0, 1}, {0.2f * c, 0, 0}};
        }
        MapDisparityTo3D::SParameter mp;
        mp.Set(uint16_t(EDisparityId::First), uint16_t(EDisparityId::Last), false, cams);
        MapDisparityTo3D::CDriver m3;
        m3.Configure(dev, f16, mp);
        CDeviceSurface pts(SImageFormat(W, H, EDataType::RGBA_Single));
        ProcessKernel(m3, pts, disp);
        auto pv = pts.CopyInto<float4>();
        const float4 pc = pv[size_t(60) * W + 100];
        float lo[3], hi[3];
        m3.GetRange(lo, hi);
        const float zw = 500.f * 0.2f / float(K);
        CHECK(std::fabs(pc.z - zw) < 1e-4f * zw && pc.w == 1.f && lo[2] <= pc.z && hi[2] >= pc.z,
              "3D: z %g (want %g), valid %g, z range %g .. %g", pc.z, zw, pc.w, lo[2], hi[2]);

        // mip-maps of the map: level 1 interior = 0.5 * code (K + 1), level 0
        // border (CannotEvaluate) = 0
        CDeviceSurfMipMap mip(f16);
        CreateDispMipMaps::CDriver mm;
        mm.Configure(dev, f16);
        CDeviceSurface tmp;
        CHECK(ThrownCode([&] { mm.Run(mip, tmp, disp, mip.MaxMipMapLevelCount() + 1); }) == CT_EINVAL,
              "mip-map level count above the maximum");
        mm.Run(mip, tmp, disp, 0);
        CHECK(mip.GetActiveMipMapLevelCount() == mip.MaxMipMapLevelCount(), "mip-map active level count");
        auto mv = mip.Surface().CopyInto<float>();
        const int mpw = mip.Surface().Format().iWidth;
        int mx = 0, my = 0;
        mip.GetOrigin(mx, my, 1);
        const float l1 = mv[size_t(my + 30) * mpw + mx + 50];
        CHECK(l1 == 0.5f * float(K + 1) && mv[0] == 0.f, "mip-map: level 1 %g, want %g; level 0 border %g", l1,
              0.5f * float(K + 1), mv[0]);

        // guided: a coarse map at half resolution holding K / 2 everywhere
        // (scaled 2 * (K / 2) = K - 1; the block ranges contain K)
        std::vector<uint8_t> coarse(size_t(W / 2) * ((H + 1) / 2), uint8_t(K / 2));
        CDeviceSurface init(SImageFormat(W / 2, (H + 1) / 2));
        init.CopyFrom(coarse.data());
        p.iUseDispInput = 1;
        BlockMatcherNCC::CDriver g;
        g.Configure(dev, fin, p);
        CHECK(ThrownCode([&] { g.Process(disp, surfL, surfR, _CDeviceSurface(), score); }) == CT_EINVAL,
              "guided NCC without a coarse map");
        ProcessKernel(g, disp, surfL, surfR, init, score);
        auto gv = disp.CopyInto<uint16_t>();
        int gbad = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) gbad += interior(x, y, 5) && gv[size_t(y) * W + x] != v[size_t(y) * W + x];
        CHECK(gbad == 0, "guided NCC: %d interior pixels differ from the full search", gbad);
    }
    {  // AW1 shifted windows, sub-pixel
        _SDisparityConfig dc;
        dc.Set(0, 64);
        BlockMatcherAW1::SParameter p;
        p.Set(dc, 0.f, 0.f, 0.f, 0, true, BlockMatcherAW1::EConfig::Shifted5_7x7,
              BlockMatcherAW1::ESimType::AbsoluteDifference);
        BlockMatcherAW1::CDriver d;
        d.Configure(dev, fin, p);
        CDeviceSurface disp(f32);
        ProcessKernel(d, disp, surfL, surfR, _CDeviceSurface(), _CDeviceSurface());
        auto v = disp.CopyInto<float>();
        int bad = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) bad += interior(x, y, 6) && !(std::fabs(v[size_t(y) * W + x] - K) < 0.5f);
        CHECK(bad == 0, "AW1: %d interior pixels not within 0.5 of %d", bad, K);

        // guided, with a coarse map at quarter resolution holding K / 4
        // (scaled 4 * (K / 4) = 4; the block ranges [0, 8] contain K)
        std::vector<uint8_t> coarse(size_t(W / 4) * (H / 4), uint8_t(K / 4));
        CDeviceSurface init(SImageFormat(W / 4, H / 4));
        init.CopyFrom(coarse.data());
        p.iUseDispInput = 1;
        BlockMatcherAW1::CDriver g;
        g.Configure(dev, fin, p);
        ProcessKernel(g, disp, surfL, surfR, init, _CDeviceSurface());
        auto gv = disp.CopyInto<float>();
        int gbad = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) gbad += interior(x, y, 6) && gv[size_t(y) * W + x] != v[size_t(y) * W + x];
        CHECK(gbad == 0, "guided AW1: %d interior pixels differ from the full search", gbad);
    }
    {  // census both ways + cross-check driver on the two maps
        _SDisparityConfig dc;
        dc.Set(0, 64);
        BlockMatcherCensus::SParameter p;
        p.xDispConfig = dc;
        BlockMatcherCensus::CDriver m;
        m.Configure(dev, fin, p);
        CDeviceSurface lr(f16), rl(f16), chk(f16), res(f16);
        _CDeviceSurface none;
        m.ProcessLR(lr, rl, chk, 1, surfL, surfR);
        CrossCheckDisparityMaps::SParameter cp;
        cp.Set(dc, 1, 1);
        CrossCheckDisparityMaps::CDriver cc;
        cc.Configure(dev, f16, cp);
        ProcessKernel(cc, res, lr, rl);
        auto a = chk.CopyInto<uint16_t>();
        auto b = res.CopyInto<uint16_t>();
        int bad = 0, differ = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const size_t i = size_t(y) * W + x;
                bad += interior(x, y, 6) && a[i] != K + 1;
                // the driver leaves the 1-pixel frame unwritten (as the reference)
                differ += x >= 1 && x < W - 1 && y >= 1 && y < H - 1 && a[i] != b[i];
            }
        CHECK(bad == 0, "census L-R: %d interior pixels not kept at d = %d", bad, K);
        CHECK(differ == 0, "ProcessLR and the cross-check driver disagree on %d pixels", differ);
        CHECK(cc.DispMin() <= K && cc.DispMax() >= K, "range %d..%d", cc.DispMin(), cc.DispMax());
        m.EnsureDeviceStatus();
        {  // two matching passes give the same three maps as the fused one
            CDeviceSurface lr2(f16), rl2(f16), chk2(f16);
            m.SetFusedLR(false);
            m.ProcessLR(lr2, rl2, chk2, 1, surfL, surfR);
            m.SetFusedLR(true);
            int d2 = 0;
            const auto p1 = lr.CopyInto<uint16_t>(), p2 = lr2.CopyInto<uint16_t>();
            const auto q1 = rl.CopyInto<uint16_t>(), q2 = rl2.CopyInto<uint16_t>();
            const auto c2 = chk2.CopyInto<uint16_t>();
            for (size_t i = 0; i < a.size(); ++i) d2 += (p1[i] != p2[i]) + (q1[i] != q2[i]) + (a[i] != c2[i]);
            CHECK(d2 == 0, "SetFusedLR(false): %d map pixels differ from the fused pass", d2);
        }

        // the same pair as a stream of frames from host memory
        CensusStream::CDriver st;
        st.Configure(dev, fin, p, 1, EDataType::UInt16);
        std::vector<std::vector<uint16_t>> frames(4, std::vector<uint16_t>(size_t(W) * H));
        int64_t last = -1;
        for (auto& fr : frames) last = st.Submit(L.data(), W, R.data(), W, fr.data(), size_t(W) * 2);
        st.Wait(last);
        int sdiff = 0;
        for (const auto& fr : frames)
            for (size_t i = 0; i < fr.size(); ++i) sdiff += fr[i] != a[i];
        CHECK(last == 3 && sdiff == 0, "stream: %d pixels differ from ProcessLR", sdiff);

        // learned confidence on the same pair: checked = winner map with
        // every pixel scoring below the threshold marked Inconsistent
        ConfidenceNet::CDriver net;
        net.Configure(dev);
        net.LoadParams(weights);
        BlockMatcherCensus::CDriver m128;
        p.xDispConfig.Set(0, 128);
        m128.Configure(dev, fin, p);
        CCurveVolume cv(W, H, 128);
        CDeviceSurface d128(f16), score(f32), checked(f16);
        m128.ProcessCurves(d128, cv, surfL, surfR);
        ProcessKernel(net, score, checked, cv, d128, 0.5f);
        auto dv = d128.CopyInto<uint16_t>();
        auto sv = score.CopyInto<float>();
        auto cvv = checked.CopyInto<uint16_t>();
        int wrong = 0, range = 0, kept = 0, n_in = 0;
        for (size_t i = 0; i < dv.size(); ++i) {
            const bool has = dv[i] >= CT_DISP_FIRST && dv[i] <= CT_DISP_LAST;
            const uint16_t want = has && sv[i] < 0.5f ? uint16_t(EDisparityId::Inconsistent) : dv[i];
            wrong += cvv[i] != want;
            range += !(sv[i] >= 0.f && sv[i] <= 1.f) && has;
            const int x = int(i % W), y = int(i / W);
            if (interior(x, y, 6)) {
                ++n_in;
                kept += cvv[i] == K + 1;
            }
        }
        CHECK(wrong == 0, "confidence: %d checked pixels disagree with the scores", wrong);
        CHECK(range == 0, "confidence: %d scores outside [0, 1]", range);
        std::printf("confidence net keeps %d of %d interior pixels of the exact shift\n", kept, n_in);
    }
    {  // batch: two pairs of different size in one call
        const int W2 = 200, H2 = 64;
        std::vector<uint8_t> L2(size_t(W2) * H2), R2(size_t(W2) * H2);
        for (int y = 0; y < H2; ++y)
            for (int x = 0; x < W2; ++x) {
                L2[size_t(y) * W2 + x] = L[size_t(y) * W + x];
                R2[size_t(y) * W2 + x] = R[size_t(y) * W + x];
            }
        CDeviceSurface sL2(SImageFormat(W2, H2)), sR2(SImageFormat(W2, H2));
        sL2.CopyFrom(L2.data());
        sR2.CopyFrom(R2.data());
        BatchStereo::CDriver b;
        b.Configure(dev, {fin, SImageFormat(W2, H2)}, {64, 32}, 1);
        CDeviceSurface o1(f16), o2(SImageFormat(W2, H2, EDataType::UInt16));
        ProcessKernel(b, std::vector<BatchStereo::SPair>{{surfL, surfR, o1}, {sL2, sR2, o2}});
        auto v1 = o1.CopyInto<uint16_t>();
        auto v2 = o2.CopyInto<uint16_t>();
        int bad = 0;
        for (int y = 6; y < H - 6; ++y)
            for (int x = K + 6; x < W - 6 - K; ++x) bad += v1[size_t(y) * W + x] != K + 1;
        for (int y = 6; y < H2 - 6; ++y)
            for (int x = K + 6; x < W2 - 6 - K; ++x) bad += v2[size_t(y) * W2 + x] != K + 1;
        CHECK(bad == 0, "batch: %d interior pixels not kept at d = %d", bad, K);
    }
    {  // a bounded device wait that runs out becomes CError(CT_ETIMEOUT), and
       // the driver keeps working afterwards
        BlockMatcherCensus::SParameter p;
        p.xDispConfig.Set(0, 64);
        BlockMatcherCensus::CDriver d;
        d.Configure(dev, fin, p);
        Ensure(ct_handle_test_wait_timeout(d.Handle(), 1024, nullptr), "test wait");
        CHECK(ThrownCode([&] { d.EnsureDeviceStatus(); }) == CT_ETIMEOUT, "timeout must surface as CT_ETIMEOUT");
        CHECK(ThrownCode([&] { d.EnsureDeviceStatus(); }) == 0, "status must be cleared after it was read");
        CDeviceSurface out(f8);
        ProcessKernel(d, out, surfL, surfR);
        auto v = out.CopyInto<uint8_t>();
        int bad = 0;
        for (int y = 5; y < H - 5; ++y)
            for (int x = K + 6; x < W - 6 - K; ++x) bad += v[size_t(y) * W + x] != K;
        CHECK(bad == 0, "census after a timeout: %d interior pixels not at d = %d", bad, K);
    }
    return g_failures;
}

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "cpu";
    int rc = 0;
    try {
        if (mode == "cpu") {
            rc = RunCpu();
        } else if (mode == "gpu" && argc > 2) {
            rc = RunGpu(argv[2]);
        } else {
            std::printf("usage: shim_test cpu | gpu <weights.f32>\n");
            return 2;
        }
    } catch (const CError& e) {
        std::printf("FAIL: uncaught CError %d: %s\n", e.Code(), e.what());
        return 1;
    }
    std::printf("%s: %s (%d failures)\n", mode.c_str(), rc ? "FAILED" : "ok", rc);
    return rc ? 1 : 0;
}
