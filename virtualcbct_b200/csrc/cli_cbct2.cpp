// vcbct_cbct2 <info txt> -- the reference's FDK program
// (Release_recon_from_forward_pro_float_CM/main.cpp) on libvcbct: reads the
// info file and flexmap, the float projections "<prefix>.<ext>"
// [V][H][W], filters them (writing "fltsngrm.raw" as the reference does),
// backprojects and writes the (short) volume [Z][N][N] to the
// reconstruction file.  The filter is the tensor-core BF16x3 one (within
// 1e-5 of the FP64 filter's scale, as the FP32 direct one is);
// VCBCT_FILTER=direct selects the FP32 direct filter.  Exit status 0 on
// success, 1 on any error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vcbct.h"

static int die(const char* what)
{
    std::fprintf(stderr, "vcbct_cbct2: %s: %s\n", what, vcbct_last_error());
    return 1;
}

static bool write_all(const char* name, const void* p, size_t size, size_t n)
{
    FILE* fp = std::fopen(name, "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(p, size, n, fp) == n;
    return (std::fclose(fp) == 0) && ok;
}

int main(int argc, char** argv)
{
    if (argc != 2) {
        std::fprintf(stderr, "\n[usage]$ vcbct_cbct2 <info filename>\n\n");
        return 1;
    }
    static vcbct_fdk_deck d;
    if (vcbct_fdk_deck_read(argv[1], &d)) return die("info file");
    // The reference opens the output first and stops if it is not writable.
    FILE* probe = std::fopen(d.recon_file, "wb");
    if (!probe) {
        std::fprintf(stderr, "ERROR: output file NOT writable\n");
        return 1;
    }
    std::fclose(probe);

    const size_t np = (size_t)d.total_proj * d.proj_height * d.proj_width;
    std::vector<float> proj(np, 0.0f), filt(np);
    char name[300];
    std::snprintf(name, sizeof name, "%s.%s", d.proj_prefix, d.proj_ext);
    FILE* fp = std::fopen(name, "rb");
    if (!fp) {
        std::fprintf(stderr, "ERROR: projection file %s NOT readable\n", name);
        return 1;
    }
    const size_t got = std::fread(proj.data(), sizeof(float), np, fp);
    std::fclose(fp);
    if (got != np) std::fprintf(stderr, "WARNING: %s holds %zu of %zu values\n", name, got, np);

    vcbct_fdk_geometry g;
    vcbct_fdk_default_geometry(&g);
    g.proj_width = d.proj_width;
    g.proj_height = d.proj_height;
    g.n_views = d.total_proj;
    g.recon_size = d.recon_size;
    g.recon_slices = d.recon_slices;
    g.zstart = d.recon_offset;
    g.recon_step = d.recon_step;
    g.recon_scale = d.recon_scale;
    g.xfactor = d.xfactor;
    g.det_pitch_iso_cm = d.det_pitch_iso_cm;
    std::fprintf(stderr, "Reconstructing z = %d to %f, Step = %f\n", d.recon_offset,
                 d.recon_offset + d.recon_slices * d.recon_step, d.recon_step);

    vcbct_fdk* f = nullptr;
    if (vcbct_fdk_create(&g, d.angles_rad, d.xshift, d.yshift, &f)) return die("fdk");
    const char* fm = std::getenv("VCBCT_FILTER");
    const int method = (fm && std::strcmp(fm, "direct") == 0) ? VCBCT_FILTER_DIRECT_F32 : VCBCT_FILTER_BF16X3;
    if (vcbct_fdk_filter(f, proj.data(), filt.data(), 0, method, nullptr)) {
        vcbct_fdk_destroy(f);
        return die("filterSinogram");
    }
    if (!write_all("fltsngrm.raw", filt.data(), sizeof(float), np)) {
        vcbct_fdk_destroy(f);
        std::fprintf(stderr, "ERROR: fltsngrm file NOT writable\n");
        return 1;
    }
    const size_t nv = (size_t)d.recon_slices * d.recon_size * d.recon_size;
    std::vector<short> vol(nv);
    if (vcbct_fdk_backproject(f, filt.data(), nullptr, vol.data(), 0, nullptr)) {
        vcbct_fdk_destroy(f);
        return die("reconstructImage");
    }
    vcbct_fdk_destroy(f);
    if (!write_all(d.recon_file, vol.data(), sizeof(short), nv)) {
        std::fprintf(stderr, "ERROR: cannot write %s\n", d.recon_file);
        return 1;
    }
    std::fprintf(stderr, "done.\n");
    return 0;
}
