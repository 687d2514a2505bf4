"""bench.py's roofline bookkeeping on the CPU: the DRAM traffic figure is tied
to a digest of the kernel sources, so the digest must cover every file that
holds a kernel of the measured cycle."""
import importlib.util
import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "arcane-benchs_b200" / "csrc"


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_digest_covers_every_cycle_kernel_source():
    bench = load_bench()
    listed = set(bench.KERNEL_SOURCES)
    for name in listed:
        assert (CSRC / name).is_file(), name
    # files defining or instantiating the cycle kernels (k_cyc_*) or the bodies
    # and helpers they inline (sweep lines, Lagrange bodies, device arithmetic)
    for f in sorted(CSRC.glob("*.cu*")):
        text = f.read_text()
        if re.search(r"\bk_cyc_\w+", text) and "__global__" in text:
            assert f.name in listed, f.name
    for f in sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")):
        assert f.name in listed, f"{f.name}: a device header the cycle kernels include"


def test_digest_is_deterministic_and_tracks_the_sources():
    bench = load_bench()
    d1, d2 = bench.kernel_sources_digest(), bench.kernel_sources_digest()
    assert d1 == d2 and re.fullmatch(r"[0-9a-f]{16}", d1)
    for key, (traffic, digest) in bench.TRAFFIC_PER_CYCLE.items():
        assert traffic > 0 and re.fullmatch(r"[0-9a-f]{16}", digest), key
        value, note = bench.cycle_traffic(key)
        # a stale figure is reported as null, a current one as the measured bytes
        assert (value is None) == (digest != d1), (key, note)
        if value is not None:
            assert value == traffic
