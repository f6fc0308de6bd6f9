// Built by tests/test_facade.py: drives the library only through the
// reference-compatible classes of include/qcstorm_b200.hpp, the way the JNI
// workers do (OnlineLocalizationLD.cpp: extract -> accumulate -> localize ->
// remove zero rows), and writes every result to files for comparison.
//
// usage: facade_check <dir>   reads  dir/para.bin (qcs_loc_para), dir/frames.bin
//                               (uint16, n_frames x H x W), dir/n_frames.txt
//                             writes dir/rois.bin, dir/wle.bin, dir/loc.bin,
//                               dir/kept.bin, dir/counts.txt
#include <cstdio>
#include <string>
#include <vector>

#include "qcstorm_b200.hpp"

static std::vector<char> slurp(const std::string &path) {
    std::vector<char> b;
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return b;
    fseek(f, 0, SEEK_END);
    b.resize(ftell(f));
    fseek(f, 0, SEEK_SET);
    if (fread(b.data(), 1, b.size(), f) != b.size()) b.clear();
    fclose(f);
    return b;
}

static void spill(const std::string &path, const void *p, size_t bytes) {
    FILE *f = fopen(path.c_str(), "wb");
    if (f) {
        fwrite(p, 1, bytes, f);
        fclose(f);
    }
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    std::vector<char> pb = slurp(dir + "/para.bin"), fb = slurp(dir + "/frames.bin"), nb = slurp(dir + "/n_frames.txt");
    if (pb.size() != sizeof(qcs_loc_para) || fb.empty() || nb.empty()) return 3;
    LocalizationPara para;
    *static_cast<qcs_loc_para *>(&para) = *reinterpret_cast<const qcs_loc_para *>(pb.data());
    const int n_frames = atoi(std::string(nb.begin(), nb.end()).c_str());
    unsigned short *frames = reinterpret_cast<unsigned short *>(fb.data());

    cudaStream_t stream;
    cudaStreamCreate(&stream);
    LDROIExtractData_TypeDef extract;
    LDLocData_TypeDef loc;
    ZeroLocalizationsRemovel_TypeDef zero;
    extract.Init(para);
    loc.Init(para);
    zero.Init();

    const int batch = LDROIExtractData_TypeDef::GetMaxBatchedNumForCurrentImageSize(para.ImageWidth, para.ImageHigh);
    const size_t frame_px = (size_t)para.ImageWidth * para.ImageHigh;
    for (int f = 0; f < n_frames; f += batch) {
        const int nb_cur = (n_frames - f) < batch ? (n_frames - f) : batch;
        extract.ExtractMolecules(frames + f * frame_px, ImageSource_CPU_Normal, para, f, nb_cur, stream);
    }
    const int n = extract.GetAccumulatedROINum();
    const int whole = para.ROISize * (para.ROISize + 1);
    spill(dir + "/rois.bin", extract.h_ImageROI, sizeof(unsigned short) * whole * n);
    spill(dir + "/wle.bin", extract.Get_h_WLEPara(), sizeof(float) * WLE_ParaNumber * n);

    loc.BFGS_MLELocalization(extract.h_ImageROI, extract.Get_h_WLEPara(), para, n, stream);
    spill(dir + "/loc.bin", loc.h_LocArry, sizeof(float) * OutParaNumGS2D * loc.oValidFluoNum);

    zero.RemoveZeroLocalizations(loc.h_LocArry, loc.oValidFluoNum, 1, extract.FirstFrame, extract.EndFrame, stream);
    spill(dir + "/kept.bin", zero.h_LocArry, sizeof(float) * OutParaNumGS2D * zero.ValidFluoNum);

    para.UpdateSRImageSize();
    ImageRenderData_TypeDef render;
    render.Init(para, 0, 0);
    render.FluoRenderTop(zero.h_LocArry, para, RenderingMode_FittedPhoton_CalculatedLocPrec, 0, zero.ValidFluoNum,
                         stream);
    std::vector<float> img((size_t)para.SRImageWidth * para.SRImageHigh);
    cudaMemcpy(img.data(), render.d_SRIntensityImg, img.size() * sizeof(float), cudaMemcpyDeviceToHost);
    spill(dir + "/render.bin", img.data(), img.size() * sizeof(float));
    render.Deinit(para);

    FILE *c = fopen((dir + "/counts.txt").c_str(), "w");
    fprintf(c, "%d %d %d %d %d %d %d\n", n, loc.oValidFluoNum, zero.ValidFluoNum, extract.FirstFrame, extract.EndFrame,
            LDLocData_TypeDef::GetFirstFrame(zero.h_LocArry, zero.ValidFluoNum),
            LDLocData_TypeDef::GetLastFrame(zero.h_LocArry, zero.ValidFluoNum));
    fclose(c);
    extract.ResetROINum();
    zero.Deinit();
    loc.Deinit(para);
    extract.Deinit();
    cudaStreamDestroy(stream);
    return 0;
}
