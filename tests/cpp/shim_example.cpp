// Drop-in use of the C++ host layer (include/aprb200.hpp): the calls below
// have the shape of LibAPR code (Example_get_apr.cpp / Example_apr_filter.cpp).
// Prints "P=<particles> sum=<sum of intensities> conv=<sum of conv output>
// recon=<sum of the piecewise-constant image> levels=<sum of the level image>
// gmag=<sum of the CFD gradient magnitude> auto_P=<particles with automatic
// parameters> grad_th=<chosen> sigma_th=<chosen>".
#include <cstdio>
#include <cstdlib>

#include "aprb200.hpp"

using namespace aprb200::compat;

int main(int argc, char **argv) {
    const char *path = argc > 1 ? argv[1] : nullptr;
    int y = 48, x = 40, z = 24;
    PixelData<uint16_t> img(y, x, z);
    if (path) {
        FILE *f = std::fopen(path, "rb");
        if (!f || std::fread(img.mesh.data(), 2, img.mesh.size(), f) != img.mesh.size()) return 2;
        std::fclose(f);
    }
    APRConverter<uint16_t> conv;
    conv.par.lambda = 3;
    conv.par.rel_error = 0.1f;
    conv.par.sigma_th = 50;
    conv.par.grad_th = 10;
    APR apr;
    if (!conv.get_apr(apr, img)) return 3;
    ParticleData<uint16_t> parts;
    parts.sample_image(apr, img);
    unsigned long long sum = 0;
    for (size_t i = 0; i < parts.size(); ++i) sum += parts[i];
    PixelData<float> st(3, 3, 3);
    for (auto &v : st.mesh) v = 1.0f / 27.0f;
    ParticleData<float> in, out;
    in.data.assign(parts.data.begin(), parts.data.end());
    APRFilter::convolve_pencil(apr, st, in, out, true, true, false);
    double cs = 0;
    for (float v : out.data) cs += v;
    PixelData<uint16_t> pc;
    APRReconstruction::reconstruct_constant(apr, pc, parts);
    PixelData<uint8_t> lv;
    APRReconstruction::reconstruct_level(apr, lv);
    unsigned long long rs = 0, ls = 0;
    for (uint16_t v : pc.mesh) rs += v;
    for (uint8_t v : lv.mesh) ls += v;
    ParticleData<float> gm;
    APRNumerics::gradient_magnitude_cfd(apr, parts, gm);
    double gs = 0;
    for (float v : gm.data) gs += v;
    // automatic parameters (APRConverter.hpp:556-561): the converter's par
    // receives the thresholds, as in the reference
    APRConverter<uint16_t> conv_auto;
    conv_auto.par = conv.par;
    conv_auto.par.auto_parameters = true;
    APR apr_auto;
    if (!conv_auto.get_apr(apr_auto, img)) return 4;
    const APRParameters used = apr_auto.get_apr_parameters();
    if (used.grad_th != conv_auto.par.grad_th || used.sigma_th != conv_auto.par.sigma_th) return 5;
    std::printf("P=%llu sum=%llu conv=%.6f recon=%llu levels=%llu gmag=%.6f auto_P=%llu grad_th=%.9g sigma_th=%.9g\n",
                (unsigned long long)apr.total_number_particles(), sum, cs, rs, ls, gs,
                (unsigned long long)apr_auto.total_number_particles(), (double)used.grad_th, (double)used.sigma_th);
    return 0;
}
