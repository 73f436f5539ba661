// SIGPROC filterbank reader and .dat/.inf writer (see sigproc.hpp).
#include "sigproc.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>

#include "errors.hpp"

namespace dedisp {
namespace sigproc {

namespace {

struct File {
    FILE* f = nullptr;
    File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode))
    {
        if (!f) DD_THROW_MSG(DEDISP_INVALID_POINTER, ("cannot open " + path).c_str());
    }
    ~File()
    {
        if (f) std::fclose(f);
    }
};

template <typename T>
T read_value(FILE* f, const char* what)
{
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1)
        DD_THROW_MSG(DEDISP_INVALID_POINTER, (std::string("truncated header at ") + what).c_str());
    return v;
}

std::string read_string(FILE* f)
{
    const int32_t n = read_value<int32_t>(f, "a string length");
    if (n < 1 || n > 4096) DD_THROW_MSG(DEDISP_INVALID_POINTER, "bad string length in header");
    std::string s((size_t)n, '\0');
    if (std::fread(&s[0], 1, (size_t)n, f) != (size_t)n)
        DD_THROW_MSG(DEDISP_INVALID_POINTER, "truncated header string");
    return s;
}

enum class Kind { Int, Double, String, Char };

// SIGPROC header keywords and their value types.
const std::map<std::string, Kind>& keywords()
{
    static const std::map<std::string, Kind> k = {
        {"telescope_id", Kind::Int}, {"machine_id", Kind::Int},    {"data_type", Kind::Int},
        {"barycentric", Kind::Int},  {"pulsarcentric", Kind::Int}, {"nbits", Kind::Int},
        {"nsamples", Kind::Int},     {"nchans", Kind::Int},        {"nifs", Kind::Int},
        {"nbeams", Kind::Int},       {"ibeam", Kind::Int},         {"npuls", Kind::Int},
        {"nbins", Kind::Int},        {"tstart", Kind::Double},     {"tsamp", Kind::Double},
        {"fch1", Kind::Double},      {"foff", Kind::Double},       {"refdm", Kind::Double},
        {"az_start", Kind::Double},  {"za_start", Kind::Double},   {"src_raj", Kind::Double},
        {"src_dej", Kind::Double},   {"period", Kind::Double},     {"fchannel", Kind::Double},
        {"source_name", Kind::String}, {"rawdatafile", Kind::String}, {"signed", Kind::Char},
    };
    return k;
}

const char* telescope_name(int id)
{
    static const char* names[] = {"Fake",   "Arecibo", "Ooty",       "Nancay", "Parkes",
                                  "Jodrell", "GBT",    "GMRT",       "Effelsberg", "ATA",
                                  "UTR-2",  "LOFAR",   "FR606",      "DE601",  "UK608"};
    return (id >= 0 && id < 15) ? names[id] : "???????";
}

const char* backend_name(int id)
{
    switch (id) {
    case 0: return "FAKE";
    case 1: return "PSPM";
    case 2: return "WAPP";
    case 3: return "AOFTM";
    case 4: return "BPP";
    case 5: return "OOTY";
    case 6: return "SCAMP";
    case 7: return "SPIGOT";
    case 10: return "ARTEMIS";
    case 11: return "Cobalt";
    default: return "????";
    }
}

}  // namespace

void read_header(const std::string& path, dedisp_b200_fil_header* h)
{
    if (!h) DD_THROW(DEDISP_INVALID_POINTER);
    std::memset(h, 0, sizeof(*h));
    h->nifs = 1;
    File file(path, "rb");
    FILE* f = file.f;
    if (read_string(f) != "HEADER_START") DD_THROW_MSG(DEDISP_INVALID_POINTER, "not a SIGPROC filterbank file");
    for (;;) {
        const std::string key = read_string(f);
        if (key == "HEADER_END") break;
        if (key == "FREQUENCY_START" || key == "FREQUENCY_END") continue;
        const auto it = keywords().find(key);
        if (it == keywords().end())
            DD_THROW_MSG(DEDISP_INVALID_POINTER, ("unknown header keyword " + key).c_str());
        switch (it->second) {
        case Kind::Int: {
            const int32_t v = read_value<int32_t>(f, key.c_str());
            if (key == "telescope_id") h->telescope_id = v;
            else if (key == "machine_id") h->machine_id = v;
            else if (key == "nbits") h->nbits = v;
            else if (key == "nchans") h->nchans = v;
            else if (key == "nifs") h->nifs = v;
            else if (key == "nbeams") h->nbeams = v;
            else if (key == "ibeam") h->ibeam = v;
            break;
        }
        case Kind::Double: {
            const double v = read_value<double>(f, key.c_str());
            if (key == "tstart") h->tstart = v;
            else if (key == "tsamp") h->tsamp = v;
            else if (key == "fch1") h->fch1 = v;
            else if (key == "foff") h->foff = v;
            else if (key == "az_start") h->az_start = v;
            else if (key == "za_start") h->za_start = v;
            else if (key == "src_raj") h->src_raj = v;
            else if (key == "src_dej") h->src_dej = v;
            break;
        }
        case Kind::String: {
            const std::string v = read_string(f);
            if (key == "source_name") {
                std::strncpy(h->source_name, v.c_str(), sizeof(h->source_name) - 1);
                h->source_name[sizeof(h->source_name) - 1] = '\0';
            }
            break;
        }
        case Kind::Char:
            (void)read_value<int8_t>(f, key.c_str());
            break;
        }
    }
    const long hdr = std::ftell(f);
    std::fseek(f, 0, SEEK_END);
    const long end = std::ftell(f);
    if (hdr < 0 || end < hdr) DD_THROW_MSG(DEDISP_INVALID_POINTER, "cannot size the data section");
    h->header_bytes = (dedisp_size)hdr;
    const size_t row = (size_t)h->nchans * (size_t)h->nifs * (size_t)h->nbits / 8;
    if (h->nchans <= 0 || h->nbits <= 0 || row == 0) DD_THROW_MSG(DEDISP_INVALID_POINTER, "header lacks nchans/nbits");
    h->nsamples = (dedisp_size)((size_t)(end - hdr) / row);
}

void read_samples(const std::string& path, const dedisp_b200_fil_header& h, size_t first, size_t count,
                  uint8_t* out)
{
    if (!out && count) DD_THROW(DEDISP_INVALID_POINTER);
    if (first + count > h.nsamples) DD_THROW_MSG(DEDISP_TOO_FEW_NSAMPS, "read past the end of the data");
    const size_t row = (size_t)h.nchans * (size_t)h.nifs * (size_t)h.nbits / 8;
    File file(path, "rb");
    if (std::fseek(file.f, (long)(h.header_bytes + first * row), SEEK_SET) != 0)
        DD_THROW_MSG(DEDISP_INVALID_POINTER, "seek failed");
    if (count && std::fread(out, row, count, file.f) != count)
        DD_THROW_MSG(DEDISP_INVALID_POINTER, "short read");
}

size_t decimate8(uint8_t* z, size_t nchans, size_t nsamps, size_t factor)
{
    if (factor <= 1) return nsamps;
    const size_t nout = nsamps / factor;
    for (size_t l = 0; l < nout; ++l) {
        for (size_t i = 0; i < nchans; ++i) {
            float acc = 0.f;
            for (size_t k = 0; k < factor; ++k) acc += (float)z[i + nchans * (l * factor + k)];
            acc /= (float)factor;
            z[i + nchans * l] = acc > 255.f ? (uint8_t)255 : (acc < 0.f ? (uint8_t)0 : (uint8_t)acc);
        }
    }
    return nout;
}

std::string dm_stem(const std::string& prefix, float dm)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "_DM%.3f", dm);
    return prefix + buf;
}

void write_dat(const std::string& prefix, float dm, const float* series, size_t n)
{
    File file(dm_stem(prefix, dm) + ".dat", "wb");
    if (n && std::fwrite(series, sizeof(float), n, file.f) != n)
        DD_THROW_MSG(DEDISP_INVALID_POINTER, "short write");
}

void write_inf(const std::string& prefix, float dm, const dedisp_b200_fil_header& h, size_t numout)
{
    const std::string stem = dm_stem(prefix, dm);
    File file(stem + ".inf", "w");
    FILE* f = file.f;
    std::fprintf(f, " Data file name without suffix          =  %s\n", stem.c_str());
    std::fprintf(f, " Telescope used                         =  %s\n", telescope_name(h.telescope_id));
    std::fprintf(f, " Instrument used                        =  %s\n", backend_name(h.machine_id));
    std::fprintf(f, " Object being observed                  =  %s\n", h.source_name);
    const int ra_h = (int)std::floor(h.src_raj / 10000.0);
    const int ra_m = (int)std::floor((h.src_raj - ra_h * 10000) / 100.0);
    const double ra_s = h.src_raj - ra_h * 10000 - ra_m * 100;
    const int dec_d = (int)std::floor(std::fabs(h.src_dej) / 10000.0);
    const int dec_m = (int)std::floor((std::fabs(h.src_dej) - dec_d * 10000) / 100.0);
    const double dec_s = std::fabs(h.src_dej) - dec_d * 10000 - dec_m * 100;
    const char sign = h.src_dej < 0.0 ? '-' : ' ';
    std::fprintf(f, " J2000 Right Ascension (hh:mm:ss.ssss)  =  %02d:%02d:%02f\n", ra_h, ra_m, ra_s);
    std::fprintf(f, " J2000 Declination     (dd:mm:ss.ssss)  = %c%02d:%02d:%s%f\n", sign, dec_d, dec_m,
                 dec_s < 10 ? "0" : "", dec_s);
    std::fprintf(f, " Data observed by                       =  Unknown\n");
    // MJD: integer part, then the fraction's digits as printed with %.15f
    char frac[64];
    std::snprintf(frac, sizeof frac, "%.15f", h.tstart - std::floor(h.tstart));
    const char* dot = std::strchr(frac, '.');
    std::fprintf(f, " Epoch of observation (MJD)             =  %d.%s\n", (int)std::floor(h.tstart),
                 dot ? dot + 1 : "0");
    std::fprintf(f, " Barycentered?           (1=yes, 0=no)  =  0\n");
    std::fprintf(f, " Number of bins in the time series      =  %d\n", (int)numout);
    std::fprintf(f, " Width of each time series bin (sec)    =  %.15g\n", h.tsamp);
    std::fprintf(f, " Any breaks in the data? (1=yes, 0=no)  =  0\n");
    std::fprintf(f, " Type of observation (EM band)          =  Radio\n");
    std::fprintf(f, " Beam diameter (arcsec)                 =  3600\n");
    std::fprintf(f, " Dispersion measure (cm-3 pc)           =  %.12g\n", dm);
    std::fprintf(f, " Central freq of low channel (Mhz)      =  %.12g\n",
                 h.fch1 - (h.nchans - 1) * std::fabs(h.foff));
    std::fprintf(f, " Total bandwidth (Mhz)                  =  %.12g\n", std::fabs(h.foff) * h.nchans);
    std::fprintf(f, " Number of channels                     =  %d\n", h.nchans);
    std::fprintf(f, " Channel bandwidth (Mhz)                =  %.12g\n", std::fabs(h.foff));
    std::fprintf(f, " Data analyzed by                       =  Unknown\n");
    std::fprintf(f, " Any additional notes:\n    Input filterbank samples have %d bits.\n", h.nbits);
}

}  // namespace sigproc
}  // namespace dedisp

// ---------------------------------------------------------------------------
// C interface (include/dedisp_b200.h)
// ---------------------------------------------------------------------------
namespace dedisp {
void note_last_error(dedisp_error code, const char* msg);
}

namespace {
template <typename F>
dedisp_error io_call(F&& fn)
{
    try {
        fn();
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        dedisp::note_last_error(e.code(), e.what());
        return e.code();
    } catch (const std::exception& e) {
        dedisp::note_last_error(DEDISP_UNKNOWN_ERROR, e.what());
        return DEDISP_UNKNOWN_ERROR;
    }
}
}  // namespace

extern "C" {

dedisp_error dedisp_b200_fil_read_header(const char* path, dedisp_b200_fil_header* header)
{
    if (!path || !header) return DEDISP_INVALID_POINTER;
    return io_call([&] { dedisp::sigproc::read_header(path, header); });
}

dedisp_error dedisp_b200_fil_read_samples(const char* path, const dedisp_b200_fil_header* header,
                                          dedisp_size first, dedisp_size count, dedisp_byte* out)
{
    if (!path || !header) return DEDISP_INVALID_POINTER;
    return io_call([&] { dedisp::sigproc::read_samples(path, *header, first, count, out); });
}

dedisp_size dedisp_b200_fil_decimate(dedisp_byte* data, dedisp_size nchans, dedisp_size nsamps,
                                     dedisp_size factor)
{
    if (!data) return 0;
    return dedisp::sigproc::decimate8(data, nchans, nsamps, factor);
}

dedisp_error dedisp_b200_write_dat(const char* prefix, dedisp_float dm, const dedisp_float* series,
                                   dedisp_size n)
{
    if (!prefix || (n && !series)) return DEDISP_INVALID_POINTER;
    return io_call([&] { dedisp::sigproc::write_dat(prefix, dm, series, n); });
}

dedisp_error dedisp_b200_write_inf(const char* prefix, dedisp_float dm, const dedisp_b200_fil_header* header,
                                   dedisp_size numout)
{
    if (!prefix || !header) return DEDISP_INVALID_POINTER;
    return io_call([&] { dedisp::sigproc::write_inf(prefix, dm, *header, numout); });
}

}  // extern "C"
