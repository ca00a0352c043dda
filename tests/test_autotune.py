"""The autotuner's selection and header output (CPU; the measurement itself
runs on the GPU: python -m disco_b200.autotune measure)."""
import os
import re
import subprocess

from disco_b200 import autotune as at
from disco_b200 import build as native


def _table():
    # ms per step per kernel for (block size, MB) candidates; each kernel has
    # its own best; 256-thread blocks are slower in total
    t = {"fp64": {(128, 4): {"k_begin": 1.0, "k_faces": 2.0, "k_update": 1.5},
                  (128, 8): {"k_begin": 0.8, "k_faces": 2.1, "k_update": 1.2},
                  (128, 16): {"k_begin": 0.9, "k_faces": 1.7, "k_update": 2.0},
                  (256, 4): {"k_begin": 0.7, "k_faces": 2.5, "k_update": 1.6}},
         "mixed": {(128, 4): {"k_begin": 0.7, "k_faces": 1.0, "k_update": 1.0},
                   (128, 8): {"k_begin": 0.9, "k_faces": 0.9, "k_update": 1.1},
                   (128, 16): {"k_begin": 0.8, "k_faces": 1.2, "k_update": 0.9},
                   (256, 4): {"k_begin": 0.1, "k_faces": 0.1, "k_update": 0.1}}}
    return t


def test_choose_per_kernel_and_precision():
    best = at.choose(_table())
    assert best["cb"] == 128                      # decided by the FP64 step
    assert best["fp64"] == {"k_begin": 8, "k_faces": 16, "k_update": 8}
    assert best["mixed"] == {"k_begin": 4, "k_faces": 8, "k_update": 16}


def test_header_defines_each_precision(tmp_path):
    res = _table()
    path = str(tmp_path / "tuned.h")
    at.write_header(res, at.choose(res), "test", path=path)
    src = open(path).read()
    # the header must select the values by translation unit
    for tu, expect in (("", {"MB_BEGIN": 8, "MB_FACES": 16, "MB_UPDATE": 8}),
                       ("-DDISCO_MIXED_TU", {"MB_BEGIN": 4, "MB_FACES": 8, "MB_UPDATE": 16})):
        cmd = ["gcc", "-E", "-dM", "-x", "c"] + ([tu] if tu else []) + [path]
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        got = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (MB_\w+) (\d+)", out)}
        assert got == expect, (tu, got)
        assert re.search(r"#define CB 128", out) and re.search(r"#define FB 128", out)
    assert "-> 16" in src


def test_committed_header_covers_every_tuned_kernel():
    src = open(at.TUNED).read()
    for macro in at.MACROS.values():
        assert src.count("#define %s " % macro) == 2, macro   # one per precision
    assert src.count("#define CB ") == 1
    assert os.path.dirname(at.TUNED) == os.path.join(native.HERE, "csrc")


def test_mhd_family_header(tmp_path):
    """The MHD family's header defines MB_MHD_* per translation unit and no
    block size (the hydro family's CB serves both)."""
    t = {"fp64": {(128, 4): {"k_flux": 3.0, "k_c2p": 2.0}, (128, 6): {"k_flux": 2.5, "k_c2p": 2.2}},
         "mixed": {(128, 4): {"k_flux": 2.0, "k_c2p": 1.0}, (128, 6): {"k_flux": 2.2, "k_c2p": 0.8}}}
    best = at.choose(t, at.MACROS_MHD)
    assert best["fp64"] == {"k_flux": 6, "k_c2p": 4} and best["mixed"] == {"k_flux": 4, "k_c2p": 6}
    path = str(tmp_path / "tuned_mhd.h")
    at.write_header(t, best, "config4_nz16", path=path, family="mhd")
    for tu, expect in (("", {"MB_MHD_FLUX": 6, "MB_MHD_C2P": 4}),
                       ("-DDISCO_MIXED_TU", {"MB_MHD_FLUX": 4, "MB_MHD_C2P": 6})):
        cmd = ["gcc", "-E", "-dM", "-x", "c"] + ([tu] if tu else []) + [path]
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        got = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (MB_\w+) (\d+)", out)}
        assert got == expect, (tu, got)
        assert not re.search(r"#define CB ", out)


def test_variant_names_per_family(tmp_path):
    assert at._parse_variant("cb128_mb6") == (128, 6)
    assert at._parse_variant("mhd_cb128_mb5", "mhd") == (128, 5)
    assert at._is_variant("mhd_cb128_mb5", "mhd") and not at._is_variant("mhd_cb128_mb5", "hydro")
    assert at._variant_dir(str(tmp_path), 128, 5, "mhd").endswith("mhd_cb128_mb5")
