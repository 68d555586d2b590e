"""Generate golden vectors by running the REFERENCE implementation's own code.

Run in a container where the reference source tree is mounted, naming it in
$SPP_REFERENCE_ROOT:

    SPP_REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_golden.py

Besides the vectors it copies the reference's small sigproc test files
(tests/data/*.fil) into tests/golden/_ref/ (kept out of version control) for
the real-file tests, which skip when the copies are absent.

It loads src/sigpyproc/core/kernels.py (numba) and single functions of
params.py / header.py / readers.py through oracle/refload.py, evaluates them
on seeded inputs and writes the outputs next to this script.  The GPU tests
and the oracle tests compare against these files; nothing at test time reads
the reference tree.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import refload  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    if not refload.available():
        raise SystemExit("reference tree not found")
    K = refload.load_kernels()
    cdd, dmc = refload.load_compute_dmdelays()
    hf = refload.load_header_freq_helpers()
    read_plan = refload.load_read_plan()

    class Hdr:
        def __init__(self, nchans, fch1, foff):
            self.nchans, self.fch1, self.foff = nchans, fch1, foff

        @property
        def chan_freqs(self):
            return hf["chan_freqs"](self)

        @property
        def ftop(self):
            return hf["ftop"](self)

        @property
        def fcenter(self):
            return hf["fcenter"](self)

        @property
        def fbottom(self):
            return hf["fbottom"](self)

        @property
        def fmax(self):
            return hf["fmax"](self)

        @property
        def fmin(self):
            return hf["fmin"](self)

    def ref_delays(nchans, fch1, foff, tsamp, dm, ref="fch1"):
        h = Hdr(nchans, fch1, foff)
        fref = float(getattr(h, ref)) if isinstance(ref, str) else float(ref)
        return cdd(h.chan_freqs, dm, tsamp, fref)

    out: dict[str, np.ndarray] = {}
    meta: dict = {"dm_constant": dmc}

    # ---- R4 unpack: the reference KAT input [7, 23] and a random byte array
    rng = np.random.default_rng(11)
    rnd = rng.integers(0, 256, size=4096, dtype=np.uint8)
    out["unpack_rand_in"] = rnd
    for nbits in (1, 2, 4):
        for order in ("big", "little"):
            fn = getattr(K, f"unpack{nbits}_8_{order}")
            for tag, arr in (("kat", np.array([7, 23], dtype=np.uint8)), ("rand", rnd)):
                u = np.empty(arr.size * 8 // nbits, dtype=np.uint8)
                fn(arr, u)
                out[f"unpack_{tag}_{nbits}_{order}"] = u

    # ---- R6 delays at the benchmark geometries and the reference test geometry
    geoms = {
        "c1": (256, 1500.0, -1.0, 64e-6, np.array([100.0])),
        "c2": (4096, 1500.0, -0.0732421875, 64e-6, 1000.0 + np.linspace(-1000.0, 1000.0, 1024)),
        "c3": (1024, 1400.0, -0.29296875, 64e-6, 500.0 + np.linspace(-500.0, 500.0, 512)),
        "c5": (4096, 1500.0, -0.0732421875, 64e-6, 1500.0 + np.linspace(-1500.0, 1500.0, 4096)),
        "parkes": (832, 4030.0, -4.0, 512e-6, np.array([0.0, 100.0, 5000.0])),
        "tutorial": (64, 1510.0, -1.09, 320e-6, np.array([10.0, 50.0, 200.0])),
    }
    meta["delays"] = {}
    for name, (nch, f1, fo, ts, dms) in geoms.items():
        for ref in ("fch1", "fcenter", "fmax", "fmin", 1234.5):
            if name in ("c2", "c5") and ref != "fch1":
                continue
            d = np.atleast_2d(ref_delays(nch, f1, fo, ts, dms, ref)).astype(np.int32)
            key = f"{name}_{ref}"
            meta["delays"][key] = {
                "geom": [nch, f1, fo, ts], "ref": ref, "ndm": int(d.shape[0]),
                "sha256": sha(d), "max": int(d.max()), "min": int(d.min()),
            }
            rows = sorted({0, min(1, d.shape[0] - 1), d.shape[0] // 2, d.shape[0] - 1})
            out[f"delays_{key}_rows"] = d[rows]
            out[f"delays_{key}_rowidx"] = np.array(rows, dtype=np.int64)
            out[f"delays_{key}_dms"] = np.asarray(dms, dtype=np.float64)
    # float (seconds) delays as the reference test geometry uses
    freqs = np.arange(1000, dtype=np.float32) * (-1.0) + 1400
    out["delays_params_sec"] = cdd(freqs, np.linspace(0, 100, 50), 0.001, freqs[0], in_samples=False)
    out["delays_params_samp"] = cdd(freqs, np.linspace(0, 100, 50), 0.001, freqs[0])

    # ---- R2 dedisperse on seeded small blocks
    rng = np.random.default_rng(12)
    u8 = rng.integers(0, 256, size=(4096, 64), dtype=np.uint8)
    out["ded_u8_in"] = u8
    for tag, dm, ref in (("dm50", 50.0, "fch1"), ("dm200", 200.0, "fch1"),
                         ("dm120_fcenter", 120.0, "fcenter")):
        d = ref_delays(64, 1510.0, -1.09, 320e-6, dm, ref).astype(np.int32)
        maxd = int(np.max(np.abs(d)))
        o = np.zeros(4096 - maxd, dtype=np.float32)
        K.dedisperse(u8.ravel(), o, d, 64, 4096, 0)
        out[f"ded_u8_{tag}_delays"] = d
        out[f"ded_u8_{tag}_out"] = o
    rng = np.random.default_rng(13)
    f32 = rng.normal(0.0, 1.0, size=(2048, 32)).astype(np.float32)
    out["ded_f32_in"] = f32
    d = ref_delays(32, 1400.0, -2.0, 256e-6, 30.0).astype(np.int32)
    o = np.zeros(2048 - int(np.max(np.abs(d))), dtype=np.float32)
    K.dedisperse(f32.ravel(), o, d, 32, 2048, 0)
    out["ded_f32_delays"] = d
    out["ded_f32_out"] = o

    # ---- R1 at config 1: the full Filterbank.dedisperse flow (read_plan blocks)
    from sigpyproc3_b200 import synth  # noqa: PLC0415

    c1 = synth.c1_filterbank(1)
    meta["c1_input_sha256"] = sha(c1)
    d = ref_delays(256, 1500.0, -1.0, 64e-6, 100.0).astype(np.int32)
    maxd = int(np.max(np.abs(d)))
    gulp = max(2 * maxd, 16384)
    tim = np.zeros(65536 - maxd, dtype=np.float32)

    class FakeFile:
        def __init__(self, raw):
            self.raw = raw
            self.pos = 0
            self.reads = []

        def seek(self, offset, whence=0):
            self.pos = offset if whence == 0 else self.pos + offset

        def creadinto(self, rbuf, ubuf=None):
            mv = memoryview(rbuf)
            n = min(len(mv), self.raw.size - self.pos)
            np.frombuffer(mv, dtype=np.uint8)[:n] = self.raw[self.pos:self.pos + n]
            self.reads.append(self.pos)
            self.pos += n
            return n

    class FakeReader:
        def __init__(self, raw, nsamples, nchans, itemsize=1):
            self.header = type("H", (), {"nsamples": nsamples, "nchans": nchans})()
            self.bitsinfo = type("B", (), {"unpack": False, "dtype": np.dtype(np.uint8)})()
            self.samp_stride = nchans * itemsize
            self.chan_stride = float(itemsize)
            self._file = FakeFile(raw)

    fr = FakeReader(c1, 65536, 256)
    for nsamps_r, ii, data in read_plan(fr, gulp=gulp, skipback=maxd, quiet=True):
        K.dedisperse(np.ascontiguousarray(data), tim, d, 256, nsamps_r, ii * (gulp - maxd))
    out["c1_tim"] = tim
    out["c1_delays"] = d

    # ---- R5 read_plan schedules (byte offsets of each read and the yielded sizes)
    plans = []
    for nsamples, nchans, gulp, start, nsamps, skip in (
        (4096, 832, 512, 0, None, 0), (4096, 832, 400, 0, None, 200), (4096, 832, 512, 0, 1024, 0),
        (65536, 256, 16384, 0, None, 1301), (10000, 64, 3000, 17, 5000, 999),
        (10000, 64, 2000, 0, None, 500), (3000, 64, 1000, 0, None, 900),
        (1000, 16, 5000, 0, None, 10),
    ):
        raw = (np.arange(nsamples * nchans) % 251).astype(np.uint8)
        fr = FakeReader(raw, nsamples, nchans)
        rec = []
        error = None
        try:
            for nsamps_r, ii, data in read_plan(fr, gulp=gulp, start=start, nsamps=nsamps,
                                                skipback=skip, quiet=True):
                rec.append([int(nsamps_r), int(ii), int(fr._file.reads[-1]),
                            sha(np.asarray(data))])
        except ValueError as exc:
            # the reference reads a full gulp for a short last block when the
            # file continues past start+nsamps, and then rejects the byte count
            error = str(exc)
        plans.append({"args": [nsamples, nchans, gulp, start, nsamps, skip], "blocks": rec,
                      "error": error})
    errs = []
    for nsamples, gulp, nsamps, skip in ((4096, 512, 1024, 1024), (4096, 512, 1024, 2000)):
        fr = FakeReader(np.zeros(nsamples * 8, np.uint8), nsamples, 8)
        try:
            list(read_plan(fr, gulp=gulp, nsamps=nsamps, skipback=skip, quiet=True))
            errs.append({"args": [nsamples, gulp, nsamps, skip], "error": None})
        except ValueError as exc:
            errs.append({"args": [nsamples, gulp, nsamps, skip], "error": str(exc)})
    meta["read_plan"] = plans
    meta["read_plan_errors"] = errs

    # ---- R3 compat: kernels.dmt_block on a float block (nchans, nsamps)
    rng = np.random.default_rng(14)
    blk = rng.normal(0, 1, size=(32, 512)).astype(np.float32)
    dmd = np.atleast_2d(ref_delays(32, 1400.0, -2.0, 256e-6, 10.0 + np.linspace(-10, 10, 16)))
    out["dmt_block_in"] = blk
    out["dmt_block_delays"] = dmd.astype(np.int64)
    out["dmt_block_out"] = K.dmt_block(blk, dmd.astype(np.int64))
    # integer-valued block (exact in float32)
    blk_i = rng.integers(0, 4, size=(32, 512)).astype(np.float32)
    out["dmt_block_int_in"] = blk_i
    out["dmt_block_int_out"] = K.dmt_block(blk_i, dmd.astype(np.int64))

    # ---- R7 kernels.subband (zero-initialised output)
    rng = np.random.default_rng(15)
    sb_in = rng.integers(0, 256, size=(2048, 64), dtype=np.uint8)
    d = ref_delays(64, 1510.0, -1.09, 320e-6, 80.0).astype(np.int32)
    maxd = int(np.max(np.abs(d)))
    c2s = (np.arange(64, dtype=np.int32) // 8).astype(np.int32)
    sb_out = np.zeros((2048 - maxd) * 8, dtype=np.float32)
    K.subband(sb_in.ravel(), sb_out, d, c2s, np.int32(maxd), np.int32(64), np.int32(8), np.int32(2048))
    out["subband_in"] = sb_in
    out["subband_delays"] = d
    out["subband_out"] = sb_out

    # ---- R10 bandpass / zero-DM / collapse, R8 downsample
    rng = np.random.default_rng(16)
    zf = rng.normal(5.0, 2.0, size=(1024, 48)).astype(np.float32)
    bp = np.zeros(48, dtype=np.float32)
    K.extract_bpass(zf.ravel(), bp, 48, 1024)
    zo = np.empty_like(zf.ravel())
    K.remove_zerodm(zf.ravel(), zo, bp, 48, 1024)
    out["zdm_in"] = zf
    out["zdm_bpass"] = bp
    out["zdm_out"] = zo.reshape(1024, 48)
    bpu = np.zeros(64, dtype=np.float32)
    K.extract_bpass(u8.ravel(), bpu, 64, 4096)
    out["bpass_u8"] = bpu
    tim = np.zeros(4096, dtype=np.float32)
    K.extract_tim(u8.ravel(), tim, 64, 4096, 0)
    out["collapse_u8"] = tim
    ds_in = rng.normal(0, 1, size=10007).astype(np.float32)
    out["ds_in"] = ds_in
    for f in (1, 2, 4, 7):
        out[f"ds_out_{f}"] = K.downsample_1d_mean(ds_in, f)

    # ---- N4 kernels.fold through the Filterbank.fold block loop (base.py:1151-1206)
    fold_cases = []
    for tag, dtype, nsamples, period, dm, accel, nbins, nints, nbands, gulp, seed in (
        ("a", np.uint8, 12000, 0.0313, 40.0, 0.0, 50, 8, 8, 2048, 21),
        ("b", np.uint8, 9000, 0.0251, 15.0, 30.0, 37, 7, 5, 1500, 22),
        ("c", np.float32, 6000, 0.0199, 25.0, -12.0, 23, 5, 6, 1024, 23),
    ):
        nch, tsamp = 64, 320e-6
        rng = np.random.default_rng(seed)
        if dtype == np.uint8:
            data_all = rng.integers(0, 256, size=nsamples * nch, dtype=np.uint8)
        else:
            data_all = rng.normal(0.0, 1.0, size=nsamples * nch).astype(np.float32)
        itemsize = np.dtype(dtype).itemsize
        fr = FakeReader(data_all.view(np.uint8), nsamples, nch, itemsize)
        fr.bitsinfo.dtype = np.dtype(dtype)
        nb = min(nbands, nch)
        cd = ref_delays(nch, 1510.0, -1.09, tsamp, dm).astype(np.int32)
        maxd = int(cd.max())
        g = max(2 * maxd, gulp)
        fold_ar = np.zeros(nbins * nints * nb, dtype=np.float32)
        count_ar = np.zeros(nbins * nints * nb, dtype=np.int32)
        for nsamps_r, ii, data in read_plan(fr, gulp=g, skipback=maxd, quiet=True):
            K.fold(np.ascontiguousarray(data), fold_ar, count_ar, cd, np.int32(maxd),
                   np.float32(tsamp), np.float32(period), np.float32(accel), np.int32(nsamples),
                   np.int32(nsamps_r), np.int32(nch), np.int32(nbins), np.int32(nints),
                   np.int32(nb), np.int32(ii * (g - maxd)))
        out[f"fold_{tag}_sum"] = fold_ar.copy()
        out[f"fold_{tag}_count"] = count_ar.copy()
        with np.errstate(divide="ignore", invalid="ignore"):
            fold_ar /= count_ar
        out[f"fold_{tag}_cube"] = fold_ar.reshape(nints, nb, nbins)
        fold_cases.append({"tag": tag, "dtype": np.dtype(dtype).name, "nsamples": nsamples,
                           "nchans": nch, "tsamp": tsamp, "fch1": 1510.0, "foff": -1.09,
                           "period": period, "dm": dm, "accel": accel, "nbins": nbins,
                           "nints": nints, "nbands": nbands, "gulp": gulp, "seed": seed,
                           "input_sha256": sha(data_all)})
    meta["fold_cases"] = fold_cases

    # ---- R9 robust z-score: np.median and the reference's _scale_iqr
    # (core/stats.py:418-502, MatchedFilter's defaults) on seeded series
    scale_iqr = refload.load_scale_iqr()
    scale_mad = refload.load_scale_mad()
    zs = []
    rng = np.random.default_rng(17)
    for k, m in enumerate((1, 2, 7, 8, 1000, 1001, 65536)):
        y = (rng.normal(3.0, 2.0, m) if k % 2 else rng.integers(0, 9, m)).astype(np.float32)
        out[f"zscore_in_{k}"] = y
        zs.append({"m": m, "median": float(np.median(y)), "iqr_scale": float(scale_iqr(y)),
                   "mad_scale": float(scale_mad(y))})
    # two thirds of the samples equal to the median: MAD 0, so the reference's
    # _scale_mad falls back to the mean absolute deviation
    y = np.full(999, 5.0, dtype=np.float32)
    y[::3] = rng.normal(5.0, 2.0, 333).astype(np.float32)
    out[f"zscore_in_{len(zs)}"] = y
    zs.append({"m": 999, "median": float(np.median(y)), "iqr_scale": float(scale_iqr(y)),
               "mad_scale": float(scale_mad(y))})
    meta["zscore"] = zs

    # ---- N2 kernels.downsample_2d_mean_flat (core/kernels.py:207-252) on
    # time-major blocks (dim1 = samples, dim2 = channels): uint8 (the mean is
    # cast back to uint8) and float32
    rng = np.random.default_rng(18)
    for tag, arr in (("u8", rng.integers(0, 256, size=(1001, 48), dtype=np.uint8)),
                     ("f32", rng.normal(0.0, 1.0, size=(1001, 48)).astype(np.float32))):
        out[f"ds2d_{tag}_in"] = arr
        for f1, f2 in ((3, 2), (4, 4), (1, 8), (7, 1)):
            out[f"ds2d_{tag}_{f1}_{f2}"] = K.downsample_2d_mean_flat(arr.ravel(), f1, f2, 1001, 48)

    # ---- N2/R10 file operations through their block loops:
    # Filterbank.remove_zerodm (base.py:961-1028: bandpass over the whole file,
    # then kernels.remove_zerodm per read_plan block, output in the input's
    # dtype) and Filterbank.downsample's per-block kernel call exactly as
    # base.py:644-653 makes it (dims passed as (nchans, nsamps_r))
    fops = {}
    for tag, nbits, nch, nsamples, seed in (("u8", 8, 64, 5000, 31), ("f32", 32, 48, 3000, 33)):
        rng = np.random.default_rng(seed)
        if nbits == 32:
            vals = rng.normal(5.0, 2.0, nsamples * nch).astype(np.float32)
        else:
            vals = rng.integers(0, 256, nsamples * nch, dtype=np.uint8)
        isz = vals.dtype.itemsize
        gulp = 1000

        def reader():
            fr = FakeReader(vals.view(np.uint8), nsamples, nch, isz)
            fr.bitsinfo.dtype = vals.dtype
            return fr

        bp = np.zeros(nch, dtype=np.float32)
        for nsamps_r, _ii, data in read_plan(reader(), gulp=16384, quiet=True):
            K.extract_bpass(np.ascontiguousarray(data), bp, nch, nsamps_r)
        zparts = []
        for nsamps_r, _ii, data in read_plan(reader(), gulp=gulp, quiet=True):
            o = np.empty(nsamps_r * nch, dtype=vals.dtype)
            K.remove_zerodm(np.ascontiguousarray(data), o, bp, nch, nsamps_r)
            zparts.append(o)
        out[f"fop_{tag}_zerodm"] = np.concatenate(zparts)
        out[f"fop_{tag}_zerodm_bpass"] = bp
        tf, ff = 4, 2
        g2 = int(np.ceil(gulp / tf) * tf)
        dparts = []
        for nsamps_r, _ii, data in read_plan(reader(), gulp=g2, quiet=True):
            dparts.append(K.downsample_2d_mean_flat(np.ascontiguousarray(data), tf, ff, nch,
                                                    nsamps_r))
        out[f"fop_{tag}_downsample_compat"] = np.concatenate(dparts)
        fops[tag] = {"nbits": nbits, "nchans": nch, "nsamples": nsamples, "gulp": gulp,
                     "tfactor": tf, "ffactor": ff, "seed": seed, "input_sha256": sha(vals)}
    meta["file_ops"] = fops

    # ---- N3 PulseExtractor window arithmetic (readers.py:393-455): the
    # reference's own property code, run on stand-in headers
    names = {"t_decimate", "disp_delay", "block_delay", "nsamps", "nstart", "nstart_file",
             "nsamps_file", "pulse_toa_block"}
    pe_src = refload._extract(refload.SRC / "readers.py", names, class_name="PulseExtractor")
    pe_ns: dict = {"np": np}
    exec(compile("from __future__ import annotations\n" + pe_src, "readers.py", "exec"), pe_ns)
    PE = type("PE", (), {n: property(pe_ns[n]) for n in names})
    pe_cases = []
    for toa, width, dm, toa_freq, nch_sub, nsamples in (
            (3000, 8, 30.0, None, None, 6000), (40, 3, 10.0, 1480.0, 16, 6000),
            (5990, 1, 50.0, None, 32, 6000), (100000, 64, 500.0, 1450.0, 40, 187520),
            (12, 0, 2.0, None, None, 900), (700, 17, 120.0, 1500.5, 8, 4096)):
        fch1, foff, tsamp, nch = 1510.0, -1.0, 320e-6, 64
        f1 = toa_freq or fch1
        nc = nch_sub or nch
        sub = Hdr(nc, f1, foff)
        e = PE()
        e.pulse_toa, e.pulse_width, e.min_nsamps = toa, width, 64
        e.sub_hdr = type("SH", (), {"nsamples": nsamples})()
        e._disp_delay = int(max(np.abs(np.atleast_1d(cdd(sub.chan_freqs, dm, tsamp, f1))))) + width * 5
        pe_cases.append({"args": [toa, width, dm, toa_freq, nch_sub, nsamples],
                         "props": {n: int(getattr(e, n)) for n in sorted(names)}})
    meta["pulse_extractor"] = pe_cases

    # ---- N3 template bank: the reference's own Template.gen_* and
    # MatchedFilter.get_box_width_spacing (core/filters.py:340-365, :508-579)
    tsrc = refload._extract(refload.SRC / "core" / "filters.py",
                            {"gen_boxcar", "gen_gaussian", "gen_lorentzian"}, class_name="Template")
    wsrc = refload._extract(refload.SRC / "core" / "filters.py", {"get_box_width_spacing"},
                            class_name="MatchedFilter")
    t_ns: dict = {"np": np, "gaussian_fwhm_to_sigma": 1.0 / (2.0 * np.sqrt(2.0 * np.log(2.0))),
                  "Template": object}
    exec(compile("from __future__ import annotations\n" + tsrc + "\n" + wsrc, "filters.py",
                 "exec"), t_ns)

    def fake_cls(arr, width, ref_bin=0, ref="start", kind="custom"):
        return arr, width, ref_bin, ref, kind

    temps = []
    for kind, widths in (("boxcar", t_ns["get_box_width_spacing"](32, 1.5)),
                         ("gaussian", np.geomspace(1, 32, int(np.ceil(np.log(32) / np.log(1.5))) + 1)),
                         ("lorentzian", np.geomspace(1, 32, int(np.ceil(np.log(32) / np.log(1.5))) + 1))):
        for k, w in enumerate(widths):
            arr, width, ref_bin, ref, kd = t_ns[f"gen_{kind}"](fake_cls, w)
            out[f"temp_{kind}_{k}"] = np.asarray(arr)
            temps.append({"kind": kind, "k": k, "width": float(width), "ref_bin": int(ref_bin),
                          "ref": ref})
    meta["templates"] = temps
    meta["box_widths_32_1p5"] = [float(w) for w in t_ns["get_box_width_spacing"](32, 1.5)]
    meta["box_widths_100_1p3"] = [float(w) for w in t_ns["get_box_width_spacing"](100, 1.3)]

    # ---- N1 real files: Filterbank.dedisperse over the reference's sigproc
    # test files -- its read_plan block loop (readers.py:171-233), its
    # unpack kernels as FileReader.creadinto applies them (io/fileio.py:284-292,
    # io/bits.py:175-182 bit orders) and kernels.dedisperse per block
    # (base.py:400-424)
    import shutil  # noqa: PLC0415

    from sigpyproc3_b200.io import sigproc as sp  # noqa: PLC0415

    refdir = HERE / "_ref"
    refdir.mkdir(exist_ok=True)
    meta["files"] = {}
    for name, dm in (("parkes_1bit", 100.0), ("parkes_2bit", 100.0), ("parkes_4bit", 100.0),
                     ("parkes_8bit_1", 100.0), ("parkes_8bit_2", 100.0),
                     ("tutorial_2bit", 30.0)):
        src = refload.TEST_DATA / f"{name}.fil"
        blob = src.read_bytes()
        hdr = sp.read_header(src)
        nbits, nch, nsamples = int(hdr["nbits"]), int(hdr["nchans"]), int(hdr["nsamples"])
        raw = np.frombuffer(blob, dtype=np.uint8)[hdr["hdrlen"]:]
        order = "little" if nbits == 1 else "big"
        unpack_fn = getattr(K, f"unpack{nbits}_8_{order}") if nbits < 8 else None

        class FileFake(FakeFile):
            def creadinto(self, rbuf, ubuf=None):
                n = super().creadinto(rbuf, ubuf)
                if unpack_fn is not None:
                    unpack_fn(np.frombuffer(memoryview(rbuf), dtype=np.uint8),
                              np.frombuffer(memoryview(ubuf), dtype=np.uint8))
                return n

        fr = FakeReader(raw, nsamples, nch)
        fr._file = FileFake(raw)
        fr.bitsinfo.unpack = nbits < 8
        fr.samp_stride = nch * nbits // 8
        fr.chan_stride = nbits / 8
        d = ref_delays(nch, float(hdr["fch1"]), float(hdr["foff"]), float(hdr["tsamp"]),
                       dm).astype(np.int32)
        maxd = int(np.max(np.abs(d)))
        gulp = max(2 * maxd, 16384)
        tim = np.zeros(nsamples - maxd, dtype=np.float32)
        for nsamps_r, ii, data in read_plan(fr, gulp=gulp, skipback=maxd, quiet=True):
            K.dedisperse(np.ascontiguousarray(data), tim, d, nch, nsamps_r, ii * (gulp - maxd))
        out[f"file_{name}_tim"] = tim
        out[f"file_{name}_delays"] = d
        meta["files"][name] = {"dm": dm, "sha256": hashlib.sha256(blob).hexdigest(),
                               "nbits": nbits, "nchans": nch, "nsamples": nsamples,
                               "maxdelay": maxd, "gulp": gulp}
        shutil.copyfile(src, refdir / f"{name}.fil")

    np.savez_compressed(HERE / "golden.npz", **out)
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1))
    print(f"wrote {len(out)} arrays, {(HERE / 'golden.npz').stat().st_size} bytes")


if __name__ == "__main__":
    main()
