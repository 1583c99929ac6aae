"""The C-ABI library loads without a GPU and exports every function include/pmg/pmg.h
declares; without a device, calls fail loudly with a status instead of falling back."""
import ctypes

import pytest

import pmg


def test_library_exports_every_declared_symbol():
    L = pmg.lib()
    names = pmg.header_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = pmg.lib()
    assert L.pmg_status_string(-5) == b"PMG_ENOCONV"
    a, b = ctypes.c_int32(), ctypes.c_int32()
    assert L.pmg_version(ctypes.byref(a), ctypes.byref(b)) == 0


def test_mesh_is_host_side_and_validates():
    m = pmg.Mesh(pmg.Box.make(coarse=(3, 2, 1), refine=2))
    assert m.n_cells() == 3 * 2 * 1 * 64
    with pytest.raises(pmg.PmgError) as e:
        pmg.Mesh(pmg.Box.make(coarse=(0, 1, 1)))
    assert e.value.status == -1


def test_null_arguments_rejected():
    L = pmg.lib()
    assert L.pmg_operator_m(None, None) == -1
    assert "NULL" in pmg.last_error()


def test_no_cpu_fallback_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(pmg.PmgError) as e:
        pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=1)), 2)
    assert e.value.status == -8


def test_new_entry_points_reject_null_arguments():
    L = pmg.lib()
    assert L.pmg_operator_dof_coordinates(None, None, None) == -1
    assert L.pmg_measure_peaks(0, 1 << 30, None) == -1
    assert "NULL" in pmg.last_error()


def test_peaks_need_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(pmg.PmgError) as e:
        pmg.measure_peaks(0, 1 << 30)
    assert e.value.status == -8
