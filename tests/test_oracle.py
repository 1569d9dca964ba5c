"""The oracle against the reference's own pins (CPU only).

- the 41 golden fixture files of the reference (tests/fixtures/p4_baseline/default), bit for bit;
- the reference's second record, of its `kspace` build (tests/fixtures/p4_baseline/kspace): the
  same 41 cases, equal to the `default` record except one f32 word in each of two files; the
  oracle's default build is within 1 ulp of that word and bit-exact elsewhere, and the oracle's
  `kspace` build (NUFFT y-stage, FFT x-stage, FFT inverse) reproduces it bit for bit;
- `restructured_forward_matches_the_literal_sum` (kspace.rs:3362-3433): rotor path vs literal sum
  to 1e-10 of peak over 16 effects x 3 geometries;
- `eddy_drive_some_reproduces_the_bvec_bval_product` (kspace.rs:3476-3504): 8 f64 bit patterns.
"""
import hashlib
import pathlib

import numpy as np
import pytest

from oracle import oracle
from tests import cases

GOLD = pathlib.Path(__file__).resolve().parent / "golden" / "p4_baseline" / "default"
GOLD_KSPACE = GOLD.parent / "kspace"


def test_fixture_files_are_the_reference_record():
    sums = dict(line.split("  ")[::-1] for line in (GOLD / "SHA256SUMS").read_text().split("\n") if line)
    assert len(sums) == 41
    for name, digest in sums.items():
        assert hashlib.sha256((GOLD / name).read_bytes()).hexdigest() == digest, name


def test_kspace_record_files_are_the_reference_record():
    sums = dict(line.split("  ")[::-1] for line in (GOLD_KSPACE / "SHA256SUMS").read_text().split("\n") if line)
    assert len(sums) == 41
    for name, digest in sums.items():
        assert hashlib.sha256((GOLD_KSPACE / name).read_bytes()).hexdigest() == digest, name


def test_kspace_record_differs_from_default_in_two_words():
    """The `kspace` build (NUFFT y-stage, FFT x-stage and inverse) agrees with the `default` build
    bit for bit except one word of `reverse` and one of `pf-contiguous-reverse` at 16x40, each a
    one-ulp difference."""
    differing = {}
    for f in sorted(GOLD.glob("*.bin")):
        a = np.fromfile(f, "<u4")
        b = np.fromfile(GOLD_KSPACE / f.name, "<u4")
        assert a.shape == b.shape, f.name
        d = np.nonzero(a != b)[0]
        if d.size:
            differing[f.stem] = d
            assert np.all(np.abs(a[d].astype(np.int64) - b[d].astype(np.int64)) <= 1), f.name
    assert sorted(differing) == ["slice-16x40o1-pf-contiguous-reverse", "slice-16x40o1-reverse"]
    assert all(d.size == 1 for d in differing.values())


def test_oracle_is_within_one_ulp_of_the_kspace_record():
    for name, bits in oracle.golden_outputs():
        want = np.fromfile(GOLD_KSPACE / f"{name}.bin", dtype="<u4")
        d = np.abs(want.astype(np.int64) - bits.astype(np.int64))
        assert d.max() <= 1, name
        assert np.count_nonzero(d) <= 1, name


def test_oracle_kspace_build_reproduces_the_kspace_record_bit_for_bit():
    """The reference's `kspace` build restated (kspace.rs:769-833 NUFFT y-stage through `Nufft1`,
    kspace.rs:1079-1123 FFT x-stage, kspace.rs:1385-1424 `inverse_2d_fft`): every word of the
    `kspace` record, including the two where it differs from the default record."""
    outs = oracle.golden_outputs(kspace=True)
    assert len(outs) == 41
    for name, bits in outs:
        want = np.fromfile(GOLD_KSPACE / f"{name}.bin", dtype="<u4")
        assert want.shape == bits.shape, name
        diff = np.nonzero(want != bits)[0]
        assert diff.size == 0, f"{name}: {diff.size} words differ"
    assert oracle.lib().oracle_kspace_build() == 0  # the default build again afterwards


def test_oracle_reproduces_the_golden_record_bit_for_bit():
    outs = oracle.golden_outputs()
    assert len(outs) == 41
    for name, bits in outs:
        want = np.fromfile(GOLD / f"{name}.bin", dtype="<u4")
        assert want.shape == bits.shape, name
        diff = np.nonzero(want != bits)[0]
        assert diff.size == 0, f"{name}: {diff.size} words differ, first at {diff[0]}"


def test_python_golden_inputs_match_the_record():
    """cases.golden_cases() (used by the GPU tests) regenerates the reference's inputs exactly."""
    for name, inp, acq in cases.golden_cases()[::6]:
        got = oracle.simulate_slice(inp, acq).view(np.uint32).ravel()
        want = np.fromfile(GOLD / f"{name}.bin", dtype="<u4")
        assert np.array_equal(got, want), name


@pytest.mark.parametrize("idx", range(48))
def test_restructured_forward_matches_the_literal_sum(idx):
    name, inp, acq, coil, ncoils = cases.literal_sum_cases()[idx]
    a = oracle.build_coil_kspace(inp, acq, coil, ncoils)
    b = oracle.reference_coil_kspace(inp, acq, coil, ncoils)
    peak = np.abs(b).max()
    worst = np.abs(a - b).max()
    assert peak > 0.0, name
    assert worst <= 1e-10 * peak, f"{name}: max |d| {worst:.3e} vs peak {peak:.3e}"


def test_eddy_known_answer_bits():
    """kspace.rs:3476-3504: the first 8 coefficients of an eddy slice, f64 bit for bit."""
    expected = [(0xbf85ec1cb1daa8d4, 0x3fa5ffff06e41c35), (0xbf3ac84a01a68680, 0x3f817f28896f61be),
                (0xbf83c1e814334026, 0xbfb080ac7ad7ff65), (0xbf7548454640584a, 0xbf8d9e9dd3358a7c),
                (0x3fb6e06347299105, 0x3fc30724fd363632), (0x3fc9ee837d7455c5, 0x3fcc89859a43e2be),
                (0x3fc5f2c7a85a66e2, 0x3fc03bf44552eb93), (0x3f8f6e71db6b4c1c, 0x3f7da1ff8d601054)]
    inp, acq = eddy_known_answer_case()
    got = oracle.build_coil_kspace(inp, acq, 0, 1).ravel()[:8]
    for i, (re, im) in enumerate(expected):
        assert (np.float64(got[i].real).view(np.uint64), np.float64(got[i].imag).view(np.uint64)) == (re, im), i


def eddy_known_answer_case():
    from mrsim_acq_b200.api import Acquisition, SliceInput, T2
    nx = ny = 16
    comp = cases.box_hires(nx, ny, 4.0, 12.0, 4.0, 12.0)
    acq = Acquisition(eddy_strength=0.05)
    bval, bvec = 1000.0, (0.6, 0.8, 0.0)
    inp = SliceInput(compartments=[comp], t2=[T2.uniform(100.0)], fmap=np.zeros(nx * ny, np.float32), sim=(nx, ny),
                     acq_matrix=(nx, ny), z=0, nz=1, eddy_drive=tuple(b * bval for b in bvec), slice_seed=7)
    return inp, acq


def test_line_timing_is_line_times_bit_for_bit():
    """kspace.rs:3337-3353: polarity alternates with ky; the table is `line_times` (restated)."""
    from mrsim_acq_b200.api import Acquisition
    for nx, ny in [(17, 70), (16, 40), (8, 9), (64, 64), (1, 1)]:
        for rev in (False, True):
            for t_line, t_echo in [(1.0, 90.0), (0.5, 30.0), (0.37, 12.0)]:
                acq = Acquisition(t_line=t_line, t_echo=t_echo, reverse_phase=rev)
                t, trf, tread, pol = oracle.line_timing(acq, nx, ny)
                # restate line_times directly (readout.rs:23-69)
                dt = t_line / nx
                half = (nx * ny) * dt / 2.0
                tt, rf, rd = np.zeros(ny), np.zeros(ny), np.zeros(ny)
                for tick in range(nx * ny):
                    x, y = tick % nx, tick // nx
                    if not rev:
                        y = ny - 1 - y
                        if y % 2 == 1:
                            x = nx - x - 1
                    elif y % 2 == 1:
                        x = nx - x - 1
                    if x == nx // 2:
                        tt[y] = dt * (tick + 0.5) - half
                        rf[y] = t_echo + tt[y]
                        rd[y] = tick * dt + dt / 2.0
                assert np.array_equal(t.view(np.uint64), tt.view(np.uint64))
                assert np.array_equal(trf.view(np.uint64), rf.view(np.uint64))
                assert np.array_equal(tread.view(np.uint64), rd.view(np.uint64))
                assert all(p == (-1 if k % 2 else 1) for k, p in enumerate(pol))
