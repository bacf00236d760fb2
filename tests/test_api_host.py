"""Host-side argument checks of the TNS mirror that run before any device
work (test/api.jl, test/backend_errors_cpu.jl, test/contracts.jl)."""
import pytest
import torch


def test_tns_defaults(ob):
    tns = ob.TNS()
    assert tns.dev == "uninitialized"
    assert tns.target_leaf_size == 32
    assert tns.refit_mode is False
    assert ob.TNS(torch.float32, ndims=2).ndims == 2


def test_radius_must_be_positive(ob):
    tns = ob.TNS()
    for bad in (-1.0, 0.0):
        with pytest.raises(ob.ArgumentError):
            ob.set_search_radius_(tns, bad)


def test_radius_is_stored_in_element_type(ob):
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.1)
    assert tns.radius == float(torch.tensor(0.1, dtype=torch.float32))


def test_dimension_mismatch(ob):
    tns = ob.TNS()
    ob.set_search_radius_(tns, 0.1)
    with pytest.raises(ob.DimensionMismatch):
        ob.add_point_set_(tns, torch.rand(2, 10))


def test_element_type_mismatch_is_a_type_error(ob):
    tns = ob.TNS(torch.float32)
    with pytest.raises(TypeError):
        ob.add_point_set_(tns, torch.rand(3, 10, dtype=torch.float64))


def test_cpu_coords_rejected_no_cpu_backend(ob):
    tns = ob.TNS()
    ob.set_search_radius_(tns, 0.1)
    with pytest.raises(ob.ArgumentError):
        ob.add_point_set_(tns, torch.rand(3, 10))


def test_run_requires_radius_and_a_set(ob):
    with pytest.raises(ob.ArgumentError):
        ob.run_(ob.TNS())
    tns = ob.TNS()
    ob.set_search_radius_(tns, 0.1)
    with pytest.raises(ob.ArgumentError):
        ob.run_(tns)


def test_device_view_requires_cuda_tns(ob):
    with pytest.raises(ob.OctopusError):
        ob.device_view(ob.TNS(), 1, 1)


def test_materialize_all_neighbors_needs_point_sets(ob):
    with pytest.raises(ob.OctopusError):
        ob.materialize_all_neighbors_(ob.TNS())


def test_build_edges_unregistered_pair(ob):
    with pytest.raises(ob.OctopusError):
        ob.build_edges_(ob.TNS(), 1, 1)


def test_colmajor_layout(ob):
    x = torch.arange(12, dtype=torch.float32).reshape(3, 4)  # row-major (3, 4)
    y = ob.colmajor(x)
    assert y.shape == (3, 4) and y.stride() == (1, 3)
    assert torch.equal(y, x)
    z = torch.rand(5, 3).t()
    assert ob.colmajor(z).data_ptr() == z.data_ptr()


def test_apply_zsort_needs_point_sets(ob):
    import torch
    with pytest.raises(ob.OctopusError):
        ob.apply_zsort(ob.TNS(), 1, torch.zeros(3))
    assert ob.prepare_zsort(ob.TNS()) is not None  # no sets: nothing to check
