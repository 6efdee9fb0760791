"""PhysicsState's constructors and dataset export on the host (no GPU).

Mirrors pySHiELD/physics_state.py: the field order and metadata of
:17-288, ``init_zeros`` (:327-343), ``init_from_storages`` (:344-364) with
an NDSL-style grid sizer, and ``xr_dataset`` (:366-383): one variable per
field, dims ``f"{dim}_{name}"``, attrs ``long_name`` and ``units``.
"""
import numpy as np
import pytest

# field names in the reference's declaration order (physics_state.py:17-288)
REFERENCE_ORDER = (
    "qvapor", "qliquid", "qice", "qrain", "qsnow", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp", "delz",
    "ua", "va", "w", "omga", "physics_updated_specific_humidity", "physics_updated_qliquid", "physics_updated_qice",
    "physics_updated_qrain", "physics_updated_qsnow", "physics_updated_qgraupel", "physics_updated_cloud_fraction",
    "physics_updated_pt", "physics_updated_ua", "physics_updated_va", "delprsi", "phii", "phil", "dz", "wmp", "prsi",
    "prsik", "land",
)
INTERFACE = ("phii", "prsi", "prsik")


def _sizer_and_factory(nx=12, ny=8, nz=10):
    from pyshield_b200.grid import GridIndexing, QuantityFactory, SubtileGridSizer

    # a 24 x 16 tile on a 2 x 2 layout: the subtile is 12 x 8
    sizer = SubtileGridSizer.from_tile_params(nx_tile=2 * nx, ny_tile=2 * ny, nz=nz, n_halo=3, extra_dim_lengths={},
                                              layout=(2, 2))
    qf = QuantityFactory(GridIndexing(nx, ny, nz), device="cpu")
    return sizer, qf


def _storages(nx, ny, nz, seed=0):
    import torch

    from pyshield_b200.physics import PhysicsState

    rng = np.random.default_rng(seed)
    out = {}
    for f in PhysicsState._state_fields():
        shape = (nx + 7, ny + 7) if f.name == "land" else (nx + 7, ny + 7, nz + 1)
        out[f.name] = torch.from_numpy(rng.normal(size=shape))
    return out


def test_field_order_and_metadata():
    import dataclasses

    from pyshield_b200.physics import PhysicsState

    names = tuple(f.name for f in PhysicsState._state_fields())
    assert names == REFERENCE_ORDER
    for f in dataclasses.fields(PhysicsState):
        if f.name in INTERFACE:
            assert f.metadata["dims"] == ["x", "y", "z_interface"]
        elif f.name == "land":
            assert f.metadata["dims"] == ["x", "y"] and f.metadata["units"] == "-"
        elif "dims" in f.metadata:
            assert f.metadata["dims"] == ["x", "y", "z"]
    meta = {f.name: f.metadata for f in PhysicsState._state_fields()}
    assert meta["pt"]["name"] == "air_temperature" and meta["pt"]["units"] == "degK"
    assert meta["qcld"]["units"] == ""
    assert meta["prsik"]["name"] == "log_interface_pressure"


def test_sizer_origin_and_extent():
    sizer, _ = _sizer_and_factory(12, 8, 10)
    assert (sizer.nx, sizer.ny, sizer.nz) == (12, 8, 10)
    assert sizer.get_origin(["x", "y", "z"]) == (3, 3, 0)
    assert sizer.get_extent(["x", "y", "z"]) == (12, 8, 10)
    assert sizer.get_extent(["x", "y", "z_interface"]) == (12, 8, 11)
    assert sizer.get_extent(["x_interface", "y_interface"]) == (13, 9)


def test_init_from_storages_wraps_in_place():
    from pyshield_b200.physics import PhysicsState

    nx, ny, nz = 12, 8, 10
    sizer, qf = _sizer_and_factory(nx, ny, nz)
    st = _storages(nx, ny, nz)
    ps = PhysicsState.init_from_storages(st, sizer=sizer, quantity_factory=qf, schemes=["GFS_microphysics"])
    for name in REFERENCE_ORDER:
        q = getattr(ps, name)
        assert q.data is st[name]
        if name == "land":
            assert q.origin == (3, 3) and q.extent == (nx, ny)
        else:
            assert q.origin == (3, 3, 0)
            assert q.extent == (nx, ny, nz + 1 if name in INTERFACE else nz)
        assert list(q.dims) == [f.metadata["dims"] for f in PhysicsState._state_fields() if f.name == name][0]
    # the microphysics state shares the quantities and owns zeroed tendencies
    m = ps.microphysics
    assert m.pt is ps.pt and m.delprsi is ps.delprsi and m.land is ps.land
    assert float(m.qv_dt.data.abs().sum()) == 0.0 and m.qv_dt.data is not m.ql_dt.data
    assert PhysicsState.init_from_storages(st, sizer, qf, schemes=[]).microphysics is None


def test_init_from_storages_needs_every_field():
    from pyshield_b200.physics import PhysicsState

    sizer, qf = _sizer_and_factory()
    st = _storages(12, 8, 10)
    del st["qo3mr"]
    with pytest.raises(KeyError):
        PhysicsState.init_from_storages(st, sizer, qf, schemes=[])


def test_init_zeros_uses_the_metadata():
    from pyshield_b200.physics import PhysicsState

    nx, ny, nz = 12, 8, 10
    _, qf = _sizer_and_factory(nx, ny, nz)
    ps = PhysicsState.init_zeros(qf, ["GFS_microphysics"])
    assert ps.phii.extent == (nx, ny, nz + 1) and ps.pt.extent == (nx, ny, nz)
    assert ps.land.extent == (nx, ny) and ps.pt.units == "degK"


def test_xr_dataset_names_dims_and_attrs():
    from pyshield_b200.physics import PhysicsState

    nx, ny, nz = 12, 8, 10
    sizer, qf = _sizer_and_factory(nx, ny, nz)
    st = _storages(nx, ny, nz, seed=3)
    ps = PhysicsState.init_from_storages(st, sizer, qf, schemes=["GFS_microphysics"])
    ds = ps.xr_dataset
    names = list(ds.data_vars)
    assert names == list(REFERENCE_ORDER)
    pt = ds["pt"]
    assert tuple(pt.dims) == ("x_pt", "y_pt", "z_pt")
    assert pt.attrs == {"long_name": "air_temperature", "units": "degK"}
    np.testing.assert_array_equal(np.asarray(pt.values), st["pt"].numpy())
    assert tuple(ds["prsi"].dims) == ("x_prsi", "y_prsi", "z_interface_prsi")
    assert tuple(ds["land"].dims) == ("x_land", "y_land")
    assert ds["qcld"].attrs["units"] == ""
    assert ds.dims["z_interface_phii"] == nz + 1 and ds.dims["x_pt"] == nx + 7
