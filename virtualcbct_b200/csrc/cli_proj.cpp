// vcbct_proj <info txt> -- the reference's projector program
// (Release_CBCT_Projection_CM/main.cpp with USE_GPU) on libvcbct: reads the
// info file, the spectrum and the x-ray DB, the flexmap and the slice window
// of the element volume, projects every view and writes "<outputname>.raw"
// (float [V][H][W]).  The x-ray DB directory is "attenuation_xraydb" in the
// current directory (prior_weight_production.cpp:333-345) unless the
// environment variable VCBCT_XRAYDB names another.  Exit status 0 on success
// (the reference exits 0 on every path), 1 on any error.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "vcbct.h"

static int die(const char* what)
{
    std::fprintf(stderr, "vcbct_proj: %s: %s\n", what, vcbct_last_error());
    return 1;
}

int main(int argc, char** argv)
{
    if (argc != 2) {
        std::fprintf(stderr, "\n[usage]$ vcbct_proj <info filename>\n\n");
        return 1;
    }
    vcbct_proj_deck d;
    if (vcbct_proj_deck_read(argv[1], &d)) return die("info file");
    std::printf("%s \n", d.spectrum);

    const char* db = std::getenv("VCBCT_XRAYDB");
    std::vector<float> mu((size_t)VCBCT_MAX_BINS * d.mat_num), pdf(VCBCT_MAX_BINS);
    int ne = 0;
    if (vcbct_attenuation_table(d.spectrum, db ? db : "attenuation_xraydb", d.mat_num, 1, mu.data(),
                                pdf.data(), &ne))
        return die("spectrum");

    const int V = d.total_proj;
    std::vector<double> ang(V, 0.0), xs(V, 0.0), ys(V, 0.0);
    int nread = 0;
    if (vcbct_flexmap_read(d.angle_file, V, ang.data(), xs.data(), ys.data(), &nread)) return die("flexmap");

    std::fprintf(stderr, "matImage num = %d, center = %d, z_reg = %f\n", d.used_slices, d.z_ic_local, d.z_reg);

    std::vector<double> c(V), s(V), xc(V), yc(V);
    if (vcbct_proj_trig_tables(d.proj_width, d.proj_height, V, ang.data(), xs.data(), ys.data(), d.det_pitch_cm,
                               d.det_pixel_num, c.data(), s.data(), xc.data(), yc.data()))
        return die("trig tables");

    vcbct_proj_geometry g{d.recon_size, d.used_slices, d.x_scale, d.z_scale, d.proj_width, d.proj_height, V,
                          d.det_pitch_cm, d.det_pitch_iso_cm, d.sad_cm, d.det_pixel_num, d.x_reg, d.y_reg,
                          d.z_reg, d.mat_num};
    vcbct_projector* p = nullptr;
    if (vcbct_projector_create(&g, c.data(), s.data(), xc.data(), yc.data(), &p)) return die("initialize");
    std::vector<float> out((size_t)V * d.proj_height * d.proj_width);
    int rc = vcbct_projector_set_spectrum(p, mu.data(), pdf.data(), ne, d.xfactor);
    int incomplete = 0;
    // slice files streamed to the GPU (reads overlap the copies and re-layout)
    if (!rc) rc = vcbct_projector_load_deck(p, &d, &incomplete, nullptr);
    if (!rc) rc = vcbct_projector_forward(p, out.data(), 0, nullptr);
    if (rc) {
        vcbct_projector_destroy(p);
        return die("projection");
    }
    vcbct_projector_destroy(p);

    char name[300];
    std::snprintf(name, sizeof name, "%s.raw", d.output_name);
    FILE* fp = std::fopen(name, "wb");
    if (!fp || std::fwrite(out.data(), sizeof(float), out.size(), fp) != out.size()) {
        if (fp) std::fclose(fp);
        std::fprintf(stderr, "vcbct_proj: cannot write %s\n", name);
        return 1;
    }
    std::fclose(fp);
    std::fprintf(stderr, "wrote %s (%d views x %d x %d)\n", name, V, d.proj_height, d.proj_width);
    return 0;
}
