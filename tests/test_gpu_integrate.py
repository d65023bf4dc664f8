"""Sector integration of beamformer results (BeamformerBase.integrate, integrate) on the device path: the
known-answer case of the reference's tests/unittests/test_integrate.py:15-142.  A rank-1 CSM of a unit
monopole at the grid point (0, 0, 1) seen by 5 seeded microphones; with 'true level' steering the map
peaks there, so the integral over any sector that holds only that point equals the map's maximum, on
every grid type and with the array and Sector forms of the region (acoular/fbeamform.py:595-685,
2435-2497; acoular/grids.py:187-209, 991-1494)."""

import numpy as np
import pytest

import acoular_b200 as ac

pytestmark = pytest.mark.gpu


def _grids():
    rect = ac.RectGrid(x_min=-1, x_max=1, y_min=-1, y_max=1, z=1, increment=1)
    return {
        'RectGrid': rect,
        'RectGrid3D': ac.RectGrid3D(x_min=-1, x_max=1, y_min=-1, y_max=1, z_min=1, z_max=1, increment=1),
        'LineGrid': ac.LineGrid(loc=(-1, 0, 1), length=2, num_points=3),
        'ImportGrid': ac.ImportGrid(pos=rect.pos),
        'MergeGrid': ac.MergeGrid(grids=[rect, ac.LineGrid(loc=(-1, 0, 1), length=2, num_points=3)]),
    }


def _sectors():
    square = [0.2, 0.2, -0.2, 0.2, -0.2, -0.2, 0.2, -0.2]
    return {
        'array2D': np.array([0, 0, 0.2]),
        'array3D': np.array([0, 0, 1, 0, 0, 1]),
        'RectSector': ac.RectSector(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2),
        'CircSector': ac.CircSector(x=0, y=0, r=0.2),
        'RectSector3D': ac.RectSector3D(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2, z_min=1, z_max=1),
        'PolySector': ac.PolySector(edges=square),
        'PolySector_ccw': ac.PolySector(edges=[0.2, -0.2, -0.2, -0.2, -0.2, 0.2, 0.2, 0.2]),
        'PolySector_open': ac.PolySector(edges=[0.2, 0.2, -0.2, 0.2, -0.2, -0.2]),
        'ConvexSector': ac.ConvexSector(edges=square),
        'MultiSector': ac.MultiSector(sectors=[ac.CircSector(x=0, y=0, r=0.2),
                                               ac.RectSector(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2),
                                               ac.PolySector(edges=square), ac.ConvexSector(edges=square)]),
    }


@pytest.fixture(scope='module')
def rank1():
    mics = ac.MicGeom(pos_total=np.random.RandomState(1).normal(size=3 * 5).reshape((3, 5)))
    f = 2000.0
    steer = ac.SteeringVector(grid=ac.ImportGrid(pos=np.array([[0.0], [0.0], [1.0]])), mics=mics)
    transf = np.empty((1, mics.num_mics, 1), dtype=complex)
    transf[0] = steer.transfer(f).T
    csm = transf @ transf.swapaxes(2, 1).conjugate()
    return mics, ac.PowerSpectraImport(csm=csm, frequencies=f), f


@pytest.mark.parametrize('sector_name', list(_sectors()))
@pytest.mark.parametrize('grid_name', list(_grids()))
def test_integrate_known_answer(rank1, grid_name, sector_name):
    mics, ps, f = rank1
    grid, sector = _grids()[grid_name], _sectors()[sector_name]
    is_array = isinstance(sector, np.ndarray)
    if is_array and grid_name in ('LineGrid', 'MergeGrid', 'ImportGrid'):
        bf = ac.BeamformerBase(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics))
        with pytest.raises(NotImplementedError):
            bf.integrate(sector)
        return
    if is_array and (grid_name == 'RectGrid3D') != (sector.shape[0] == 6):
        pytest.skip('array sectors: 2-D regions on 2-D grids, 3-D boxes on 3-D grids')
    bf = ac.BeamformerBase(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics))
    res = bf.synthetic(f)
    integ = ac.integrate(data=res, sector=sector, grid=grid)
    assert np.shape(integ) == ()
    assert integ == res.max()
    got = bf.integrate(sector)
    assert got.shape == (1,)
    assert got[0] == res.max()
    # many rows at once: each row summed over the sector's points
    data = np.random.RandomState(2).rand(3, grid.size)
    ind = grid.subdomain(sector) if isinstance(sector, ac.Sector) else grid.indices(*sector)
    rows = ac.integrate(data=data, sector=sector, grid=grid)
    assert rows.shape == (3,)
    for i in range(3):
        assert np.isclose(rows[i], data[i].reshape(grid.shape)[ind].sum())


def test_empty_sectors_select_nothing():
    """Sectors away from the grid with no border and no nearest-point fallback select no point."""
    grid = ac.RectGrid(x_min=-1, x_max=1, y_min=-1, y_max=1, z=1, increment=1)
    off = 10.0
    kw = {'include_border': False, 'default_nearest': False}
    for sec in (ac.RectSector(x_min=off - 0.2, x_max=off + 0.2, y_min=off - 0.2, y_max=off + 0.2, **kw),
                ac.CircSector(x=off, y=off, r=0.2, **kw),
                ac.PolySector(edges=[off + 0.2, off + 0.2, off - 0.2, off + 0.2, off - 0.2, off - 0.2], **kw)):
        assert not sec.contains(grid.pos).any()
        assert ac.integrate(data=np.ones(grid.size), sector=sec, grid=grid) == 0.0
