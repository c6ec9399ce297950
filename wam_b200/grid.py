"""Grid-module arrays of a regular latitude-longitude grid.

Builds what the reference pre-processor writes for a non-reduced grid
(preproc_module.f90:2128-2193 geometry, :2285-2363 sea-point numbering and
neighbour tables, wam_coordinate_module.f90:706-746 periodicity): sea points
numbered south to north, west to east within a row; KLAT(IJ,1|2,1|2) the
south/north neighbour (closest and second closest, equal on a regular grid),
KLON(IJ,1|2) the west/east neighbour, 0 for land; WLAT = 1.
Angles are integer 1/100 arc-seconds (M_SEC) as in the reference.
"""
import numpy as np

M_DEGREE = 360000
M_S_PER = 360 * M_DEGREE
_RAD = np.float32(np.float32(3.1415927) / np.float32(180.0))
_CIRC = np.float32(40000000.0)


def regular_grid(mask, south_deg, west_deg, dlat_deg, dlon_deg):
    """mask[nx, ny] True = sea (i = longitude index, k = latitude index)."""
    mask = np.asarray(mask, dtype=bool)
    nx, ny = mask.shape
    amosop = int(round(south_deg * M_DEGREE))
    amowep = int(round(west_deg * M_DEGREE))
    xdella = int(round(dlat_deg * M_DEGREE))
    xdello = int(round(dlon_deg * M_DEGREE))
    amoeap = amowep + (nx - 1) * xdello
    iper = abs(amowep - amoeap - xdello + M_S_PER) <= nx // 2
    # geometry in REAL precision
    k = np.arange(ny)
    xlat = (np.float32(1) * (amosop + k * xdella)).astype(np.float32) / np.float32(M_DEGREE) * _RAD
    sinph = np.sin(xlat.astype(np.float32)).astype(np.float32)
    cosph = np.cos(xlat.astype(np.float32)).astype(np.float32)
    delphi = np.float32(xdella) / np.float32(M_DEGREE) * _CIRC / np.float32(360.0)
    if iper:
        zdello = int(round((amoeap - amowep + xdello) / nx))
    else:
        zdello = int(round((amoeap - amowep) / (nx - 1)))
    dellam = np.full(ny, np.float32(zdello) / np.float32(M_DEGREE) * _CIRC / np.float32(360.0), np.float32)
    # sea-point numbering: rows south to north, west to east (1-based)
    order = mask.T  # (ny, nx)
    num = np.zeros((ny, nx), np.int64)
    flat = order.ravel()
    num.ravel()[flat] = np.arange(1, flat.sum() + 1)
    nsea = int(flat.sum())
    kk, ii = np.nonzero(order)  # row-major: k outer, i inner, matches numbering
    ip = num[kk, ii]
    klon = np.zeros((2, nsea), np.int32)
    west = np.where(ii > 0, num[kk, np.maximum(ii - 1, 0)], num[kk, nx - 1] if iper else 0)
    east = np.where(ii < nx - 1, num[kk, np.minimum(ii + 1, nx - 1)], num[kk, 0] if iper else 0)
    if not iper:
        west = np.where(ii > 0, west, 0)
        east = np.where(ii < nx - 1, east, 0)
    klon[0] = west
    klon[1] = east
    south = np.where(kk > 0, num[np.maximum(kk - 1, 0), ii], 0)
    north = np.where(kk < ny - 1, num[np.minimum(kk + 1, ny - 1), ii], 0)
    klat = np.zeros((2, 2, nsea), np.int32)  # [j][ic][ij]
    klat[0, 0] = south
    klat[0, 1] = north
    klat[1] = klat[0]
    assert (ip == np.arange(1, nsea + 1)).all()
    return dict(nsea=nsea, nx=nx, ny=ny, iper=int(iper), klat=klat.ravel(), klon=klon.ravel(),
                wlat=np.ones(2 * nsea, np.float32), kfromij=(kk + 1).astype(np.int32), ixlg=(ii + 1).astype(np.int32),
                kxlt=(kk + 1).astype(np.int32), sinph=sinph, cosph=cosph, dellam=dellam, delphi=float(delphi),
                amosop=amosop, amowep=amowep, amoeap=amoeap, xdella=xdella, xdello=xdello,
                lat=south_deg + k * dlat_deg)
