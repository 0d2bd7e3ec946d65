"""CPU tests of the product's CSV writers against the oracle's restatement of the Fortran
edit descriptors (src/PT.f90:318-341)."""
import numpy as np
import pytest

VALUES = [(-2.5, 0.0, 1.5, 400.0), (0.5, -0.25, 0.1, 20000.0), (1.2345, -0.9999, 0.00004, 612.34567),
          (-0.0001, 2.0, -1.0, 1234.5678)]


@pytest.mark.parametrize("J,D,B,T", VALUES)
def test_file_tag_matches_oracle(oracle, ib, J, D, B, T):
    want = "_".join([oracle.fmt_F0(J, 4), oracle.fmt_F0(D, 4), oracle.fmt_F0(B, 4), oracle.fmt_E0(T, 4)])
    assert ib.pt_file_tag(J, D, B, T) == want


@pytest.mark.parametrize("J,D,B,T", VALUES)
def test_pt_data_record_bytes(oracle, ib, tmp_path, J, D, B, T):
    wm, sk, ws, m = -0.98765, 3, 0.0123, np.array([0.1, -0.25, 0.995])
    path = tmp_path / "data.csv"
    ib.write_pt_data_csv(str(path), J, D, B, T, wm, sk, ws, m)
    part1 = ",".join([oracle.fmt_F0(J, 4), oracle.fmt_F0(D, 4), oracle.fmt_F0(B, 4), oracle.fmt_F0(T, 10)]) + ","
    part2 = ",".join([oracle.fmt_F0(wm, 4), oracle.fmt_I0m(sk, 4), oracle.fmt_F0(ws, 2)] +
                     [oracle.fmt_F0(v, 2) for v in m])
    want = ("J,D,B,T,winding_number_middle,skyrmion_number_middle,winding_number_spread,sx,sy,sz\n" +
            part1 + part2.ljust(500) + "\n\n")
    assert path.read_bytes() == want.encode()


def test_pt_data_readable_by_consumers(ib, tmp_path):
    """The record parses as the analysis scripts read it (pandas, whitespace stripped)."""
    import pandas as pd
    path = tmp_path / "data.csv"
    ib.write_pt_data_csv(str(path), -1.0, 0.5, 0.2, 400.0, -1.0, 1, 0.002, [0.0, 0.1, 0.9])
    df = pd.read_csv(path, na_values="********")
    assert list(df.columns) == ["J", "D", "B", "T", "winding_number_middle", "skyrmion_number_middle",
                                "winding_number_spread", "sx", "sy", "sz"]
    row = df.iloc[0]
    assert row["J"] == -1.0 and row["D"] == 0.5 and row["T"] == 400.0 and row["sz"] == 0.9


def test_formatters_agree_on_many_values(oracle, ib):
    rng = np.random.default_rng(3)
    for v in np.concatenate([rng.normal(size=200) * 10, [0.0, -0.0, 1e-9, -1e-9, 0.99995, -0.99995]]):
        tag = ib.pt_file_tag(float(v), 0.0, 0.0, 1.0)
        assert tag.split("_")[0] == oracle.fmt_F0(float(v), 4)


def test_frame_filename_and_info(ib, tmp_path):
    """Frame names as write(frame_filename, '(A,A,I5.5,A)') forms them (src/ISING.f90:218), and
    info.txt read back the way the visualisation scripts parse it
    (skyrmion_evolution_simple.py:86-91, visualise_skyrmion.py:15-20)."""
    assert ib.frame_filename("./out   ", 7) == "./out/frame_00007.csv"
    assert ib.frame_filename("o", 99999) == "o/frame_99999.csv"
    assert ib.frame_filename("o", 100000) == "o/frame_*****.csv"
    assert ib.frame_filename("o", -1) == "o/frame_*****.csv"
    path = tmp_path / "info.txt"
    for frames, cells, a in ((41, 16, 2.8), (1, 128, 1.0), (3, 96, 0.05), (0, 8, 3.5e9)):
        ib.write_frame_info(str(path), frames, cells, a)
        lines = path.read_text().splitlines(True)
        assert len(lines) == 2
        assert int(lines[0].strip()) == frames
        mesh_params = lines[1].strip().split()
        assert int(mesh_params[0]) == cells
        assert float(mesh_params[1]) == pytest.approx(float(np.float32(a)), rel=1e-8)
