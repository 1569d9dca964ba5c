"""Copy the reference crate's golden record into this repository.

The reference (Rust `mrsim-acq`) pins its 2D EPI path with 44 little-endian f32 fixture files,
written by `tests/golden_baseline.rs:28-142` of the reference crate: 39 per-slice cases
(interleaved re, im of the Roemer-combined image) and 2 series cases (magnitude then phase),
once for the `default` build (twiddle-table x-stage, direct inverse DFT) and once for the `kspace`
build (NUFFT y-stage, FFT x-stage, FFT inverse).  The reference cannot be run in this image (no
Rust toolchain), so these files are the oracle's only end-to-end pin.  They are data, copied
unchanged, so the parity tests can run where the reference tree is absent.

Usage:  python tests/golden/copy_reference_fixtures.py REFERENCE_ROOT
"""
import hashlib
import pathlib
import shutil
import sys

DST = pathlib.Path(__file__).resolve().parent / "p4_baseline"


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: copy_reference_fixtures.py REFERENCE_ROOT (the reference crate's root directory)")
    src = pathlib.Path(sys.argv[1]) / "tests" / "fixtures" / "p4_baseline"
    for build in ("default", "kspace"):
        out = DST / build
        out.mkdir(parents=True, exist_ok=True)
        lines = []
        for f in sorted((src / build).glob("*.bin")):
            shutil.copyfile(f, out / f.name)
            lines.append(f"{hashlib.sha256(f.read_bytes()).hexdigest()}  {f.name}")
        (out / "SHA256SUMS").write_text("\n".join(lines) + "\n")
        print(f"{build}: {len(lines)} files")


if __name__ == "__main__":
    main()
