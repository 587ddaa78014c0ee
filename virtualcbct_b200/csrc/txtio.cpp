// txtio.cpp -- the reference's input decks: the projector's and the FDK's
// info files (txt), flexmaps and the per-slice element volume files.
//
// Field order and scanf formats follow loadData of
// Release_CBCT_Projection_CM/projectionData.cpp:63-102 and
// Release_recon_from_forward_pro_float_CM/projectionDataMVkV.cpp:51-97; the
// derived quantities follow the same files' loadProjectionData.  Host code
// only: nothing here touches the GPU.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace {

using vcbct::fail;

constexpr double kPi = 3.141592653589793238462643383279;  // physParams.h:1

// physParams.h:47-51 of the projector ("400 dete", CM units)
constexpr double kDetPitchCm = 0.05;
constexpr double kDetPitchIsoCm = 0.032509752;
constexpr double kSadCm = 100.0;
constexpr double kDetPixelNum = 800.0;
constexpr double kDetIsoCm = 53.8;
// R/physParams.h:24-25
constexpr double kFdkPitchIsoKv = 0.032509752;
constexpr double kFdkPitchIsoMv = 0.032509752;

// A deck reader: every field is "two lines skipped, then one value line",
// after a six-line header.  A file that ends early leaves the value line
// empty, which the reference then parses as nothing (the field keeps its
// previous content); here that is an error.
class Deck {
public:
    explicit Deck(const char* path) : fp_(std::fopen(path, "r")) {}
    ~Deck()
    {
        if (fp_) std::fclose(fp_);
    }
    bool ok() const { return fp_ != nullptr; }
    bool skip(int n)
    {
        for (int i = 0; i < n; i++)
            if (!std::fgets(buf_, sizeof buf_, fp_)) return false;
        return true;
    }
    // Returns the value line of the next field, or nullptr at end of file.
    const char* field()
    {
        if (!skip(2)) return nullptr;
        if (!std::fgets(buf_, sizeof buf_, fp_)) return nullptr;
        return buf_;
    }

private:
    FILE* fp_;
    char buf_[512];  // LINEBUF_SIZE
};

int field_error(const char* path, const char* name)
{
    return fail(VCBCT_ERR_IO, std::string(path) + ": missing or unreadable field '" + name + "'");
}

// sscanf("%s") into a fixed buffer, bounded.
template <size_t Cap>
bool read_word(const char* line, char (&dst)[Cap])
{
    char fmt[16];
    std::snprintf(fmt, sizeof fmt, "%%%zus", Cap - 1);
    return std::sscanf(line, fmt, dst) == 1;
}

}  // namespace

extern "C" int vcbct_flexmap_read(const char* path, int capacity, double* angles_rad, double* xshift,
                                  double* yshift, int* n_entries)
{
    if (!path || capacity < 0 || !n_entries || (capacity > 0 && (!angles_rad || !xshift || !yshift)))
        return fail(VCBCT_ERR_ARG, "invalid argument");
    FILE* fp = std::fopen(path, "r");
    if (!fp) return fail(VCBCT_ERR_IO, std::string("angle data file: ") + path + " not found");
    int n = 0;
    for (;;) {
        double a, x, y;
        char cls[16];
        const int r = std::fscanf(fp, "%lf %lf %lf %15s", &a, &x, &y, cls);
        if (r == EOF) break;
        if (r != 4) {
            std::fclose(fp);
            return fail(VCBCT_ERR_IO, std::string(path) + ": malformed flexmap entry " + std::to_string(n + 1));
        }
        if (n >= capacity) {
            std::fclose(fp);
            return fail(VCBCT_ERR_LIMIT, std::string(path) + ": more flexmap entries than " +
                                             std::to_string(capacity));
        }
        angles_rad[n] = a * kPi / 180.0;
        xshift[n] = x;
        yshift[n] = y;
        n++;
    }
    std::fclose(fp);
    *n_entries = n;
    return VCBCT_OK;
}

extern "C" int vcbct_proj_deck_read(const char* path, vcbct_proj_deck* d)
{
    if (!path || !d) return fail(VCBCT_ERR_ARG, "NULL argument");
    std::memset(d, 0, sizeof *d);
    Deck f(path);
    if (!f.ok()) return fail(VCBCT_ERR_IO, std::string("info file: ") + path + " not found");
    if (!f.skip(6)) return fail(VCBCT_ERR_IO, std::string(path) + ": header shorter than 6 lines");
    const char* l;
#define VC_FIELD(name, expr)                         \
    if (!(l = f.field()) || !(expr)) return field_error(path, name)
    VC_FIELD("spectrum", read_word(l, d->spectrum));
    VC_FIELD("total projections", std::sscanf(l, "%d", &d->total_proj) == 1);
    VC_FIELD("projection width", std::sscanf(l, "%d", &d->proj_width) == 1);
    VC_FIELD("projection height", std::sscanf(l, "%d", &d->proj_height) == 1);
    VC_FIELD("angle data file", read_word(l, d->angle_file));
    VC_FIELD("material image prefix", read_word(l, d->mat_prefix));
    VC_FIELD("IC z position", std::sscanf(l, "%d", &d->z_ic) == 1);
    VC_FIELD("output name", read_word(l, d->output_name));
    VC_FIELD("scale", std::sscanf(l, "%lf %lf %lf", &d->x_scale, &d->y_scale, &d->z_scale) == 3);
    VC_FIELD("input size", std::sscanf(l, "%d", &d->recon_size) == 1);
    VC_FIELD("num of slices", std::sscanf(l, "%d", &d->recon_slices) == 1);
    VC_FIELD("mat_num", std::sscanf(l, "%d", &d->mat_num) == 1);
    VC_FIELD("material type", read_word(l, d->mat_type));
    VC_FIELD("density factor", std::sscanf(l, "%lf", &d->xfactor) == 1);
    VC_FIELD("image shift", std::sscanf(l, "%lf %lf %lf", &d->x_reg, &d->y_reg, &d->z_reg_file) == 3);
#undef VC_FIELD
    d->det_pitch_cm = kDetPitchCm;
    d->det_pitch_iso_cm = kDetPitchIsoCm;
    d->sad_cm = kSadCm;
    d->det_pixel_num = kDetPixelNum;
    d->det_iso_cm = kDetIsoCm;
    if (d->total_proj <= 0 || d->proj_width <= 0 || d->proj_height <= 0 || d->recon_size <= 0 ||
        d->recon_slices <= 0 || d->mat_num <= 0 || d->z_scale <= 0.0)
        return fail(VCBCT_ERR_ARG, std::string(path) + ": sizes must be positive");
    if (d->mat_num > VCBCT_MAX_MATERIALS) return fail(VCBCT_ERR_LIMIT, "mat_num above VCBCT_MAX_MATERIALS");

    // Slice window around the isocentre that the cone reaches
    // (projectionData.cpp:173-185); reconSize/2 is an integer division.
    const double z_length = (d->sad_cm + (d->recon_size / 2) * d->y_scale) / (d->det_iso_cm + d->sad_cm) *
                            d->det_pitch_cm * d->det_pixel_num;
    const int iz_length = (int)(z_length / d->z_scale);
    int linemin = d->z_ic - (iz_length / 2 + 1);
    int linemax = d->z_ic + (iz_length / 2 + 1);
    if (linemin < 0) linemin = 0;
    if (linemax >= d->recon_slices) linemax = d->recon_slices;
    d->slice_first = linemin;
    d->used_slices = linemax > linemin ? linemax - linemin : 0;
    if (d->used_slices <= 0) return fail(VCBCT_ERR_ARG, std::string(path) + ": empty slice window");
    d->z_ic_local = d->z_ic - linemin;
    // main.cpp:103 (integer division of the slice count)
    d->z_reg = (double)(d->used_slices / 2 - d->z_ic_local) * d->z_scale;
    return VCBCT_OK;
}

extern "C" int vcbct_proj_deck_load_volume(const vcbct_proj_deck* d, uint16_t* volume, int* n_incomplete)
{
    if (!d || !volume) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (d->used_slices <= 0 || d->recon_size <= 0 || d->mat_num <= 0)
        return fail(VCBCT_ERR_ARG, "deck has no slice window (call vcbct_proj_deck_read)");
    const size_t slice = (size_t)d->recon_size * d->recon_size * d->mat_num;
    std::vector<uint16_t> pixels(slice, 0);  // reused across slices, as the reference's buffer
    int bad = 0;
    char name[600];
    for (int t = 0; t < d->used_slices; t++) {
        std::snprintf(name, sizeof name, "%s_%03d.raw", d->mat_prefix, d->slice_first + t);
        FILE* fp = std::fopen(name, "rb");
        if (!fp) {
            std::fprintf(stderr, "data file: %s not found\n", name);
            bad++;
        } else {
            const size_t got = std::fread(pixels.data(), 1, slice * sizeof(uint16_t), fp);
            std::fclose(fp);
            if (got != slice * sizeof(uint16_t)) {
                std::fprintf(stderr, "WARNING: pixel data size unmatch (%s)\n", name);
                bad++;
            }
        }
        std::memcpy(volume + (size_t)t * slice, pixels.data(), slice * sizeof(uint16_t));
    }
    if (n_incomplete) *n_incomplete = bad;
    return VCBCT_OK;
}

extern "C" int vcbct_fdk_deck_read(const char* path, vcbct_fdk_deck* d)
{
    if (!path || !d) return fail(VCBCT_ERR_ARG, "NULL argument");
    std::memset(d, 0, sizeof *d);
    Deck f(path);
    if (!f.ok()) return fail(VCBCT_ERR_IO, std::string("info file: ") + path + " not found");
    if (!f.skip(6)) return fail(VCBCT_ERR_IO, std::string(path) + ": header shorter than 6 lines");
    const char* l;
#define VC_FIELD(name, expr)                         \
    if (!(l = f.field()) || !(expr)) return field_error(path, name)
    VC_FIELD("energy label", read_word(l, d->energy_class));
    VC_FIELD("total projections", std::sscanf(l, "%d", &d->total_proj) == 1);
    VC_FIELD("projection width", std::sscanf(l, "%d", &d->proj_width) == 1);
    VC_FIELD("projection height", std::sscanf(l, "%d", &d->proj_height) == 1);
    VC_FIELD("projection header bytes", std::sscanf(l, "%d", &d->proj_header_bytes) == 1);
    VC_FIELD("projection file", read_word(l, d->proj_prefix));
    VC_FIELD("file number digits", std::sscanf(l, "%d", &d->proj_num_digits) == 1);
    const bool kv = std::strcmp(d->energy_class, "kV") == 0;
    const bool mv = std::strcmp(d->energy_class, "MV") == 0;
    if (!kv && !mv)
        return fail(VCBCT_ERR_ARG, std::string(path) + ": energy label must be kV or MV");
    // The first-file-number field is unused by the float path; an unparsable
    // value (the shipped decks write "hore") leaves it at 0.
    if (!(l = f.field())) return field_error(path, "first file number");
    if (std::sscanf(l, kv ? "%X" : "%d", &d->proj_first_number) != 1) d->proj_first_number = 0;
    d->det_pitch_iso_cm = kv ? kFdkPitchIsoKv : kFdkPitchIsoMv;
    VC_FIELD("projection extension", read_word(l, d->proj_ext));
    VC_FIELD("angle data file", read_word(l, d->angle_file));
    VC_FIELD("reconstruction size", std::sscanf(l, "%d", &d->recon_size) == 1);
    VC_FIELD("target class", read_word(l, d->target_class));
    VC_FIELD("reconstruction start z", std::sscanf(l, "%d", &d->recon_offset) == 1);
    VC_FIELD("reconstruction z step", std::sscanf(l, "%lf", &d->recon_step) == 1);
    VC_FIELD("reconstruction slices", std::sscanf(l, "%d", &d->recon_slices) == 1);
    VC_FIELD("reconstruction scale", std::sscanf(l, "%lf", &d->recon_scale) == 1);
    VC_FIELD("CT value factor", std::sscanf(l, "%d", &d->xfactor) == 1);
    VC_FIELD("reconstruction file", read_word(l, d->recon_file));
#undef VC_FIELD
    if (d->total_proj <= 0 || d->proj_width <= 0 || d->proj_height <= 0 || d->recon_size <= 0)
        return fail(VCBCT_ERR_ARG, std::string(path) + ": sizes must be positive");
    if (d->total_proj > VCBCT_FDK_MAX_VIEWS)
        return fail(VCBCT_ERR_LIMIT, "more projections than VCBCT_FDK_MAX_VIEWS");

    // Flexmap with the class filter (projectionDataMVkV.cpp:159-177).
    FILE* fp = std::fopen(d->angle_file, "r");
    if (!fp) return fail(VCBCT_ERR_IO, std::string("angle data file: ") + d->angle_file + " not found");
    std::vector<double> pa, px, py;
    std::vector<char> keep;
    double first = 0.0, thirtieth = 0.0;
    for (;;) {
        double a, x, y;
        char cls[16];
        const int r = std::fscanf(fp, "%lf %lf %lf %15s", &a, &x, &y, cls);
        if (r == EOF) break;
        if (r != 4) {
            std::fclose(fp);
            return fail(VCBCT_ERR_IO, std::string(d->angle_file) + ": malformed flexmap entry");
        }
        if ((int)pa.size() >= VCBCT_FDK_MAX_VIEWS) {
            std::fclose(fp);
            return fail(VCBCT_ERR_LIMIT, "flexmap longer than VCBCT_FDK_MAX_VIEWS");
        }
        if (pa.empty()) first = a;
        if (pa.size() == 29) thirtieth = a;
        pa.push_back(a);
        px.push_back(x);
        py.push_back(y);
        keep.push_back(std::strcmp(d->target_class, "*") == 0 || std::strcmp(cls, d->target_class) == 0);
    }
    std::fclose(fp);
    const int nl = (int)pa.size();
    d->n_lines = nl;
    // Reversed when the 1st angle minus the 30th is negative (:180-211).
    d->reversed = (nl >= 30 && first - thirtieth < 0.0) ? 1 : 0;
    int nt = 0;
    double xsum = 0.0;
    for (int i = 0; i < nl; i++) {
        const int src = d->reversed ? nl - 1 - i : i;
        if (!keep[src]) continue;
        if (nt >= d->total_proj) return fail(VCBCT_ERR_LIMIT, "more matching flexmap entries than projections");
        d->angles_rad[nt] = pa[src] * kPi / 180.0;
        d->xshift[nt] = px[src];
        d->yshift[nt] = py[src];
        xsum += px[src];
        nt++;
    }
    d->n_target = nt;
    // Panel offset class from the mean xshift (:276-281); NaN (no entries)
    // falls through to "M" as in the reference.
    const double xavg = xsum / nt;
    std::snprintf(d->panel_class, sizeof d->panel_class, "%s", xavg < 6 ? "S" : (xavg > 15 ? "L" : "M"));

    // Slice-count correction (:283-302): z in cm against the height in pixels.
    if (d->recon_step > 0 && d->recon_offset + d->recon_step * (d->recon_slices - 1) >= d->proj_height)
        d->recon_slices = (int)((d->proj_height - d->recon_offset) / d->recon_step);
    else if (d->recon_step < 0 && d->recon_offset + d->recon_step * (d->recon_slices - 1) < 0)
        d->recon_slices = (int)((d->recon_offset + 1) / (-d->recon_step));
    if (d->recon_slices <= 0) return fail(VCBCT_ERR_ARG, std::string(path) + ": no reconstruction slices");
    return VCBCT_OK;
}
