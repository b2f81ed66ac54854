"""The autotuner's table file (zfmm_autotune_save / load) on the host: a
loaded table is written back unchanged, and a malformed file is refused
without touching the table."""
from zfmm_b200 import _capi


def test_table_file_roundtrip(tmp_path):
    L = _capi.lib()
    f = tmp_path / "tune.txt"
    f.write_text("k_hl2t 21 0 64\nk_tab_m2l 20 0 128\n")
    n0 = L.zfmm_autotune_entries()
    assert L.zfmm_autotune_load(str(f).encode()) == 0
    assert L.zfmm_autotune_entries() == n0 + 2
    g = tmp_path / "back.txt"
    assert L.zfmm_autotune_save(str(g).encode()) == 0
    lines = set(g.read_text().split("\n")) - {""}
    assert {"k_hl2t 21 0 64", "k_tab_m2l 20 0 128"} <= lines
    bad = tmp_path / "bad.txt"
    bad.write_text("k_hl2t 21 0 64\nk_hp2p 5 0 100\n")  # 100 is not a multiple of 32
    assert L.zfmm_autotune_load(str(bad).encode()) == 1
    assert L.zfmm_autotune_entries() == n0 + 2
    assert L.zfmm_autotune_load(str(tmp_path / "missing.txt").encode()) == 1
