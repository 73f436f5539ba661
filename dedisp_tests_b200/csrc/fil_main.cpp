// dedisp_fil: dedisperse a SIGPROC filterbank file and write one .dat/.inf
// pair per DM trial, with the options of the reference's tdd_fil /
// dedisp_fil / fdd_fil programs (bin/fil/fil.hpp:55-303) and a plan chosen
// by -k (tdd, dedisp or fdd) instead of one program per plan.
#include <getopt.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <vector>

#include "dedisp/DedispPlan.hpp"
#include "dedisp_b200.h"
#include "fdd/FDDGPUPlan.hpp"
#include "tdd/TDDPlan.hpp"

namespace {

void usage()
{
    std::printf(
        "Usage: dedisp_fil -f <file> [-k tdd|dedisp|fdd] -D [GPU device] -r [DM start,end] -s [DM step]\n\n"
        "-f <FILE file>      SIGPROC filterbank file to read as input\n"
        "-k <plan>           tdd (default), dedisp or fdd\n"
        "-o <output prefix>  Output prefix\n"
        "-D [GPU device]     GPU device number to use (default: 0)\n"
        "-r [DM start(,end)] Start (and end) values of DM range to dedisperse (default: 0,50)\n"
        "-s [DM step]        Linear DM step (with -n); without it DM trials follow generate_dm_list\n"
        "-n [ntrials]        Number of DM trials (with -s)\n"
        "-d [decimate]       Decimate timeseries by this factor (8-bit input; default: 1)\n"
        "-N [samples]        Number of samples to write (default: all)\n"
        "-w [pulse width]    Expected intrinsic pulse width for optimal DM trials (default: 4.0us)\n"
        "-t [tolerance]      Smearing tolerance factor between DM trials (default: 1.25)\n"
        "-q                  Quiet; no information to screen\n"
        "-h                  This help\n");
}

}  // namespace

int main(int argc, char* argv[])
{
    std::string filename, prefix = "test", kind = "tdd";
    int device = 0, verbose = 1, arg;
    float dm_start = 0.f, dm_end = 50.f, dm_step = 0.f, pulse_width = 4.f, tol = 1.25f;
    size_t ndec = 1, dm_count = 0, numout = 0;
    if (argc < 2) {
        usage();
        return 0;
    }
    while ((arg = getopt(argc, argv, "f:k:D:hr:s:w:t:qo:d:n:N:")) != -1) {
        switch (arg) {
        case 'f': filename = optarg; break;
        case 'k': kind = optarg; break;
        case 'o': prefix = optarg; break;
        case 'r':
            if (std::strchr(optarg, ',')) std::sscanf(optarg, "%f,%f", &dm_start, &dm_end);
            else dm_start = (float)std::atof(optarg);
            break;
        case 's': dm_step = (float)std::atof(optarg); break;
        case 'd': ndec = (size_t)std::atol(optarg); break;
        case 'n': dm_count = (size_t)std::atol(optarg); break;
        case 'N': numout = (size_t)std::atol(optarg); break;
        case 'D': device = std::atoi(optarg); break;
        case 'w': pulse_width = (float)std::atof(optarg); break;
        case 't': tol = (float)std::atof(optarg); break;
        case 'q': verbose = 0; break;
        default: usage(); return 0;
        }
    }
    if (filename.empty()) {
        std::fprintf(stderr, "No input file (-f)\n");
        return 1;
    }
    dedisp_b200_fil_header h;
    if (dedisp_b200_fil_read_header(filename.c_str(), &h) != DEDISP_NO_ERROR) {
        char msg[256];
        dedisp_b200_last_error(msg, sizeof msg);
        std::fprintf(stderr, "Error reading %s: %s\n", filename.c_str(), msg);
        return 1;
    }
    if (h.nifs != 1) {
        std::fprintf(stderr, "Wrong number of polarizations (not 1). Exiting.\n");
        return 1;
    }
    if (ndec > 1 && h.nbits != 8) {
        std::fprintf(stderr, "Decimation needs 8-bit input. Exiting.\n");
        return 1;
    }
    const size_t row = (size_t)h.nchans * h.nbits / 8;
    std::vector<uint8_t> input(h.nsamples * row);
    std::clock_t c0 = std::clock();
    if (dedisp_b200_fil_read_samples(filename.c_str(), &h, 0, h.nsamples, input.data()) != DEDISP_NO_ERROR) {
        std::fprintf(stderr, "Error reading the data of %s\n", filename.c_str());
        return 1;
    }
    size_t nsamp = h.nsamples;
    if (ndec > 1) {
        nsamp = dedisp_b200_fil_decimate(input.data(), (dedisp_size)h.nchans, nsamp, ndec);
        h.tsamp *= (double)ndec;
        h.nsamples = nsamp;
    }
    if (verbose) {
        std::printf("Frequency of highest channel              : %f MHz\n", h.fch1);
        std::printf("Bandwidth                                 : %f MHz\n", std::fabs(h.foff) * h.nchans);
        std::printf("Number of channels (channel width)        : %d (%f MHz)\n", h.nchans, std::fabs(h.foff));
        std::printf("Sample time                               : %f us\n", h.tsamp * 1e6);
        std::printf("Observation duration                      : %f s (%zu samples)\n", h.tsamp * nsamp, nsamp);
        std::printf("Number of polarizations/bit depth         : %d/%d\n", h.nifs, h.nbits);
        std::printf("Reading input took %.2f seconds\n", (double)(std::clock() - c0) / CLOCKS_PER_SEC);
    }

    std::unique_ptr<dedisp::Plan> plan;
    try {
        if (kind == "tdd") plan.reset(new dedisp::TDDPlan(h.nchans, (float)h.tsamp, (float)h.fch1, (float)h.foff, device));
        else if (kind == "dedisp") plan.reset(new dedisp::DedispPlan(h.nchans, (float)h.tsamp, (float)h.fch1, (float)h.foff, device));
        else if (kind == "fdd") plan.reset(new dedisp::FDDGPUPlan(h.nchans, (float)h.tsamp, (float)h.fch1, (float)h.foff, device));
        else {
            std::fprintf(stderr, "Unknown plan %s\n", kind.c_str());
            return 1;
        }
        if (dm_step > 0.f && dm_count > 0) {
            std::vector<float> dms(dm_count);
            for (size_t i = 0; i < dm_count; ++i) dms[i] = dm_start + dm_step * (float)i;
            plan->set_dm_list(dms.data(), dm_count);
        } else {
            plan->generate_dm_list(dm_start, dm_end, pulse_width, tol);
        }
        const size_t ndm = plan->get_dm_count(), md = plan->get_max_delay();
        if (nsamp < md) {
            std::fprintf(stderr, "Too few samples (%zu) for the maximum delay (%zu)\n", nsamp, md);
            return 1;
        }
        auto* fdd = dynamic_cast<dedisp::FDDGPUPlan*>(plan.get());
        if (fdd) {  // time series output, like the TDD plans
            dedisp::FddOptions o;
            o.segmented = 1;
            o.output = dedisp::FddOutput::TimeSeries;
            fdd->set_options(o);
        }
        const size_t nout = nsamp - md;
        const float* dmlist = plan->get_dm_list();
        if (verbose) {
            std::printf("Computing %zu DMs from %f to %f pc/cm^3\n", ndm, dmlist[0], dmlist[ndm - 1]);
            std::printf("Max DM delay is %zu samples (%f seconds)\n", md, md * h.tsamp);
            std::printf("Computing %zu out of %zu total samples\n", nout, nsamp);
        }
        std::vector<float> output(ndm * nout);
        c0 = std::clock();
        plan->execute(nsamp, input.data(), h.nbits, reinterpret_cast<uint8_t*>(output.data()), 32, 0);
        if (verbose) std::printf("Dedispersion took %.2f seconds\n", (double)(std::clock() - c0) / CLOCKS_PER_SEC);
        size_t nw = (numout == 0 || numout > nout) ? nout : numout;
        if (nw % 2) --nw;  // an even count, as the reference writes
        for (size_t i = 0; i < ndm; ++i) {
            if (dedisp_b200_write_dat(prefix.c_str(), dmlist[i], output.data() + i * nout, nw) != DEDISP_NO_ERROR ||
                dedisp_b200_write_inf(prefix.c_str(), dmlist[i], &h, nw) != DEDISP_NO_ERROR) {
                std::fprintf(stderr, "Error writing the output of DM %f\n", dmlist[i]);
                return 1;
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "Error: %s\n", e.what());
        return 1;
    }
    return 0;
}
