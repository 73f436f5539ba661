"""SIGPROC filterbank reader and .dat/.inf writer (host-side, through the C
ABI), and the dedisp_fil tool on a GPU."""
import math
import os
import struct
import subprocess

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy


def _s(x: str) -> bytes:
    return struct.pack("<i", len(x)) + x.encode()


def write_fil(path, data, nchans, nbits, tsamp=64e-6, fch1=1500.0, foff=-0.5, tstart=60000.123456,
              source="J0000+0000", extra=b""):
    hdr = _s("HEADER_START")
    hdr += _s("rawdatafile") + _s("synthetic.raw")
    hdr += _s("source_name") + _s(source)
    hdr += _s("telescope_id") + struct.pack("<i", 4)
    hdr += _s("machine_id") + struct.pack("<i", 10)
    hdr += _s("data_type") + struct.pack("<i", 1)
    hdr += _s("src_raj") + struct.pack("<d", 123456.78)
    hdr += _s("src_dej") + struct.pack("<d", -451203.5)
    hdr += _s("az_start") + struct.pack("<d", 12.5)
    hdr += _s("za_start") + struct.pack("<d", 33.25)
    hdr += _s("tstart") + struct.pack("<d", tstart)
    hdr += _s("tsamp") + struct.pack("<d", tsamp)
    hdr += _s("fch1") + struct.pack("<d", fch1)
    hdr += _s("foff") + struct.pack("<d", foff)
    hdr += _s("nchans") + struct.pack("<i", nchans)
    hdr += _s("nbits") + struct.pack("<i", nbits)
    hdr += _s("nifs") + struct.pack("<i", 1)
    hdr += _s("nbeams") + struct.pack("<i", 13)
    hdr += _s("ibeam") + struct.pack("<i", 2)
    hdr += _s("signed") + struct.pack("<b", 0)
    hdr += extra
    hdr += _s("HEADER_END")
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(np.ascontiguousarray(data).tobytes())
    return len(hdr)


def test_header_and_samples(tmp_path):
    rng = np.random.default_rng(1)
    nchans, nsamps = 64, 1000
    data = rng.integers(0, 256, (nsamps, nchans), dtype=np.uint8)
    path = str(tmp_path / "a.fil")
    hbytes = write_fil(path, data, nchans, 8)
    h = dd.fil_read_header(path)
    assert (h.nchans, h.nbits, h.nifs, h.nsamples, h.header_bytes) == (nchans, 8, 1, nsamps, hbytes)
    assert (h.tsamp, h.fch1, h.foff, h.tstart) == (64e-6, 1500.0, -0.5, 60000.123456)
    assert (h.telescope_id, h.machine_id, h.nbeams, h.ibeam) == (4, 10, 13, 2)
    assert h.source_name == b"J0000+0000"
    h2, rows = dd.fil_read(path, 100, 50)
    assert np.array_equal(rows, data[100:150])
    # packed 2-bit data: sample count from the data size
    packed = sy.pack(rng.integers(0, 4, (800, 128), dtype=np.uint32), 2)
    path2 = str(tmp_path / "b.fil")
    write_fil(path2, packed, 128, 2)
    h3, rows3 = dd.fil_read(path2)
    assert h3.nsamples == 800 and np.array_equal(rows3, packed)


def test_bad_files(tmp_path):
    path = str(tmp_path / "bad.fil")
    with open(path, "wb") as f:
        f.write(_s("NOT_A_HEADER"))
    with pytest.raises(dd.DedispError):
        dd.fil_read_header(path)
    path2 = str(tmp_path / "unk.fil")
    write_fil(path2, np.zeros((10, 32), np.uint8), 32, 8, extra=_s("mystery") + struct.pack("<i", 7))
    with pytest.raises(dd.DedispError):
        dd.fil_read_header(path2)
    with pytest.raises(dd.DedispError):
        dd.fil_read_header(str(tmp_path / "missing.fil"))


def test_decimate_matches_reference_rule():
    """Mean over `factor` consecutive samples per channel, float, truncated
    to a byte (bin/fil/fil.hpp:31-52)."""
    rng = np.random.default_rng(2)
    nchans, nsamps, factor = 48, 1003, 4
    data = rng.integers(0, 256, (nsamps, nchans), dtype=np.uint8)
    work = data.copy()
    n = dd.fil_decimate(work, nchans, factor)
    assert n == nsamps // factor
    blocks = data[: n * factor].astype(np.float32).reshape(n, factor, nchans)
    acc = np.zeros((n, nchans), np.float32)
    for k in range(factor):
        acc = acc + blocks[:, k, :]
    want = np.clip(acc / np.float32(factor), 0, 255).astype(np.uint8)
    assert np.array_equal(work[:n], want)


def _expected_inf(stem, dm, h, numout):
    ra_h = math.floor(h.src_raj / 10000.0)
    ra_m = math.floor((h.src_raj - ra_h * 10000) / 100.0)
    ra_s = h.src_raj - ra_h * 10000 - ra_m * 100
    dec_d = math.floor(abs(h.src_dej) / 10000.0)
    dec_m = math.floor((abs(h.src_dej) - dec_d * 10000) / 100.0)
    dec_s = abs(h.src_dej) - dec_d * 10000 - dec_m * 100
    frac = ("%.15f" % (h.tstart - math.floor(h.tstart))).split(".")[1]
    lines = [
        " Data file name without suffix          =  %s" % stem,
        " Telescope used                         =  %s" % "Parkes",
        " Instrument used                        =  %s" % "ARTEMIS",
        " Object being observed                  =  %s" % h.source_name.decode(),
        " J2000 Right Ascension (hh:mm:ss.ssss)  =  %02d:%02d:%02f" % (ra_h, ra_m, ra_s),
        " J2000 Declination     (dd:mm:ss.ssss)  = %c%02d:%02d:%s%f" % (
            "-" if h.src_dej < 0 else " ", dec_d, dec_m, "0" if dec_s < 10 else "", dec_s),
        " Data observed by                       =  Unknown",
        " Epoch of observation (MJD)             =  %d.%s" % (math.floor(h.tstart), frac),
        " Barycentered?           (1=yes, 0=no)  =  0",
        " Number of bins in the time series      =  %d" % numout,
        " Width of each time series bin (sec)    =  %.15g" % h.tsamp,
        " Any breaks in the data? (1=yes, 0=no)  =  0",
        " Type of observation (EM band)          =  Radio",
        " Beam diameter (arcsec)                 =  3600",
        " Dispersion measure (cm-3 pc)           =  %.12g" % np.float32(dm),
        " Central freq of low channel (Mhz)      =  %.12g" % (h.fch1 - (h.nchans - 1) * abs(h.foff)),
        " Total bandwidth (Mhz)                  =  %.12g" % (abs(h.foff) * h.nchans),
        " Number of channels                     =  %d" % h.nchans,
        " Channel bandwidth (Mhz)                =  %.12g" % abs(h.foff),
        " Data analyzed by                       =  Unknown",
        " Any additional notes:",
        "    Input filterbank samples have %d bits." % h.nbits,
    ]
    return "\n".join(lines) + "\n"


def test_dat_and_inf_writer(tmp_path):
    path = str(tmp_path / "c.fil")
    write_fil(path, np.zeros((10, 32), np.uint8), 32, 8)
    h = dd.fil_read_header(path)
    prefix = str(tmp_path / "out")
    series = np.arange(11, dtype=np.float32) * 0.5
    dm = 12.345678
    dd.write_dat_inf(prefix, dm, series, h)
    stem = prefix + "_DM%.3f" % np.float32(dm)
    assert np.array_equal(np.fromfile(stem + ".dat", np.float32), series)
    assert open(stem + ".inf").read() == _expected_inf(stem, dm, h, series.size)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tdd", "dedisp", "fdd"])
def test_dedisp_fil_tool(tmp_path, kind):
    """The command-line tool writes the plan's dedispersed series per DM."""
    rng = np.random.default_rng(3)
    nchans, nsamps = 256, 20000
    data = rng.integers(0, 256, (nsamps, nchans), dtype=np.uint8)
    path = str(tmp_path / "d.fil")
    write_fil(path, data, nchans, 8, tsamp=64e-6, fch1=1500.0, foff=-0.5)
    prefix = str(tmp_path / "res")
    r = subprocess.run([dd.fil_tool_path(), "-f", path, "-k", kind, "-r", "0", "-s", "2.5", "-n", "9",
                        "-o", prefix, "-q"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    dms = (np.float32(0) + np.float32(2.5) * np.arange(9, dtype=np.float32)).astype(np.float32)
    cls = {"tdd": dd.TDDPlan, "dedisp": dd.DedispPlan, "fdd": dd.FDDGPUPlan}[kind]
    p = cls(nchans, np.float32(64e-6), np.float32(1500.0), np.float32(-0.5))
    p.set_dm_list(dms)
    if kind == "fdd":
        p.set_options(segmented=1, timeseries=True)
    nout = nsamps - p.get_max_delay()
    want = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, data, 8, want, 32)
    nw = nout - (nout % 2)
    for i, dm in enumerate(dms):
        stem = prefix + "_DM%.3f" % dm
        got = np.fromfile(stem + ".dat", np.float32)
        assert got.size == nw
        if kind == "fdd":
            assert np.allclose(got, want[i, :nw], rtol=0, atol=1e-5 * np.abs(want).max())
        else:
            assert np.array_equal(got.view(np.uint32), want[i, :nw].view(np.uint32))
        assert os.path.exists(stem + ".inf")
