"""kukan restart files (rw_wfpot8f.F90): the record layout gfortran writes
for write_wf / write_rhovht, written out byte by byte here from the Fortran
source, and round trips through the readers."""
import struct

import numpy as np
import pytest

from rspacedist_b200 import checkpoint as CK


def rec(data: bytes) -> bytes:
    return struct.pack("<i", len(data)) + data + struct.pack("<i", len(data))


def test_file_names():
    assert CK.fname("wfc", 0, 0) == "wfc.00000.000"
    assert CK.fname("wfc", 12, 3) == "wfc.00012.003"
    assert CK.fname("rho", 7) == "rho.00007"
    with pytest.raises(ValueError):
        CK.fname("wfc", 100000, 0)


def test_wfc_layout_and_round_trip(tmp_path):
    shape = (4, 3, 2)
    N = 24
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((5, N))
    sval = np.array([-0.5, -0.2, 0.1, 0.3, 0.7])
    path = CK.write_wf(str(tmp_path), psi, sval, shape)
    raw = open(path, "rb").read()
    # write(20) wfc_version / nrc,nums,ncol,neigmx,numk,ncpx,ncpy,ncpz /
    # nrx,nry,nrz,myr_kpt / ksym / sval / svecre(:,:,:,l,1,1) for l = 1..neigmx
    want = (rec(struct.pack("<i", 5)) + rec(struct.pack("<8i", 0, 1, 1, 5, 1, 4, 3, 2)) +
            rec(struct.pack("<4i", 0, 0, 0, 0)) + rec(struct.pack("<i", 0)) +
            rec(sval.astype("<f8").tobytes()) +
            b"".join(rec(psi[l].astype("<f8").tobytes()) for l in range(5)))
    assert raw == want
    sv, back = CK.read_wf(str(tmp_path), 5, shape)
    assert np.array_equal(sv, sval) and np.array_equal(back, psi)
    sv3, back3 = CK.read_wf(str(tmp_path), 3, shape)  # fewer states than the file holds
    assert np.array_equal(sv3, sval[:3]) and np.array_equal(back3, psi[:3])
    with pytest.raises(ValueError):
        CK.read_wf(str(tmp_path), 6, shape)  # 'not enough eigenstates'
    with pytest.raises(ValueError):
        CK.read_wf(str(tmp_path), 5, (4, 3, 3))  # 'unexpected array dimensions'


def test_fp32_bands_widen_and_round(tmp_path):
    import torch
    shape = (4, 4, 4)
    psi = torch.randn(3, 64, dtype=torch.float32)
    CK.write_wf(str(tmp_path), psi, [0.0, 1.0, 2.0], shape)
    out = torch.empty(3, 64, dtype=torch.float32)
    CK.read_wf(str(tmp_path), 3, shape, out=out)
    assert torch.equal(out, psi)


def test_rho_and_vht_layout(tmp_path):
    shape = (2, 2, 2)
    rho = np.arange(8, dtype=np.float64) * 0.25
    path = CK.write_rho(str(tmp_path), rho, shape)
    raw = open(path, "rb").read()
    # rho_version / nspv,ncpx,ncpy,ncpz,nradmx,npoint,num_atcell / nrx,nry,nrz /
    # na_atcell,natcell_inf / rhosmt / rhotrur(:,:,:,1:0) / rhosmtr(:,:,:,1:0)
    want = (rec(struct.pack("<i", 3)) + rec(struct.pack("<7i", 1, 2, 2, 2, 1, 1, 0)) +
            rec(struct.pack("<3i", 0, 0, 0)) + rec(struct.pack("<i", 0)) +
            rec(rho.astype("<f8").tobytes()) + rec(b"") + rec(b""))
    assert raw == want
    got = CK.read_rho(str(tmp_path), shape)
    assert np.array_equal(got[0], rho) and got[1] == []
    assert CK.read_rho(str(tmp_path), shape, name="r_o") is None
    vh = np.linspace(-1, 1, 64)
    path = CK.write_vht(str(tmp_path), vh, shape)
    raw = open(path, "rb").read()
    want = (rec(struct.pack("<i", 3)) + rec(struct.pack("<4i", 2, 2, 2, 2)) +
            rec(struct.pack("<3i", 0, 0, 0)) + rec(vh.astype("<f8").tobytes()))
    assert raw == want
    assert np.array_equal(CK.read_vht(str(tmp_path), shape), vh)


def test_subrecords(tmp_path, monkeypatch):
    # records beyond the subrecord limit are split; shrink the limit to test it
    monkeypatch.setattr(CK, "_MAX_SUB", 16)
    p = tmp_path / "sub.bin"
    data = bytes(range(40))
    with open(p, "wb") as f:
        CK.write_record(f, data)
        CK.write_record(f, b"tail")
    raw = p.read_bytes()
    want = (struct.pack("<i", -16) + data[:16] + struct.pack("<i", 16) +
            struct.pack("<i", -16) + data[16:32] + struct.pack("<i", -16) +
            struct.pack("<i", 8) + data[32:] + struct.pack("<i", -8) + rec(b"tail"))
    assert raw == want
    with open(p, "rb") as f:
        assert CK.read_record(f) == data
        assert CK.read_record(f) == b"tail"
