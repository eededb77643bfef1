"""Host-side geometry of the equiangular gnomonic cubed sphere (numpy).

Panel p holds the reference's blockID p + 1; a point of a panel has the
equiangular coordinates (x2, x3) in [-pi/4, pi/4] and the gnomonic
coordinates X = tan(x2), Y = tan(x3).  Used by the shell problem generator
and by tests; the device path builds its own tables.

    latlon(block_id, X, Y)          CubedSphere::GetLatLon (cubed_sphere.cpp:94-106)
    vec_abp_from_rll / vec_rll_from_abp   cubed_sphere_transform.cpp:11-61
    rll_from_xyp                    cubed_sphere_transform.cpp:63-120
"""
import numpy as np

from ._abi import NGHOST


def panel_angles(nside):
    """equiangular faces and centres of one panel, ghosts included"""
    n = nside + 2 * NGHOST
    d = np.pi / 2.0 / nside
    xf = -np.pi / 4.0 + (np.arange(n + 1) - NGHOST) * d
    xv = 0.5 * (xf[1:] + xf[:-1])
    return xf, xv


def cos_theta(X, Y):
    """cosine of the angle between the panel's x2 and x3 coordinate lines"""
    return -X * Y / (np.sqrt(1.0 + X * X) * np.sqrt(1.0 + Y * Y))


def rll_from_xyp(dX, dY, nP):
    """longitude, latitude of gnomonic point (dX, dY) on panel index nP"""
    dX = np.asarray(dX, dtype=np.float64)
    dY = np.asarray(dY, dtype=np.float64)
    if nP in (1, 3, 5, 2):
        off = {1: 0.0, 3: 0.5 * np.pi, 5: np.pi, 2: 1.5 * np.pi}[nP]
        lon = np.arctan(dX) + off
        lat = np.arctan(dY / np.sqrt(1.0 + dX * dX))
    elif nP == 0:
        lon = np.where(np.abs(dX) > 1e-10, np.arctan2(dX, -dY), np.where(dY <= 0.0, 0.0, np.pi))
        lat = 0.5 * np.pi - np.arctan(np.sqrt(dX * dX + dY * dY))
    else:  # 4
        lon = np.where(np.abs(dX) > 1e-10, np.arctan2(dX, dY), np.where(dY > 0.0, 0.0, np.pi))
        lat = -0.5 * np.pi + np.arctan(np.sqrt(dX * dX + dY * dY))
    lon = np.where(lon < 0.0, lon + 2.0 * np.pi, lon)
    return lon, lat


def latlon(block_id, X, Y):
    """(lat, lon) of the panel point with gnomonic coordinates (X, Y)"""
    lon, lat = rll_from_xyp(Y, -X, block_id - 1)
    return lat, 2.0 * np.pi - lon


def xyz(block_id, X, Y):
    """unit position vector of a panel point"""
    lat, lon = latlon(block_id, X, Y)
    return np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])


def vec_abp_from_rll(X, Y, block_id, U, V):
    C = np.sqrt(1 + X * X)
    D = np.sqrt(1 + Y * Y)
    E = np.sqrt(X * X + Y * Y)
    delta = np.sqrt(1 + X * X + Y * Y)
    if block_id in (2, 3, 4, 6):
        return X * Y / delta * U - V, C * D / delta * U
    if block_id == 1:
        return (-D * Y / (delta * E) * U - D * X / E * V,
                C * X / (delta * E) * U - C * Y / E * V)
    return (D * Y / (delta * E) * U + D * X / E * V,
            -C * X / (delta * E) * U + C * Y / E * V)


def vec_rll_from_abp(X, Y, block_id, V2, V3):
    C = np.sqrt(1 + X * X)
    D = np.sqrt(1 + Y * Y)
    E = np.sqrt(X * X + Y * Y)
    delta = np.sqrt(1 + X * X + Y * Y)
    if block_id in (2, 3, 4, 6):
        return delta / (C * D) * V3, X * Y / (C * D) * V3 - V2
    if block_id == 1:
        return (-delta * Y / (D * E) * V2 + delta * X / (C * E) * V3,
                -X / (D * E) * V2 - Y / (C * E) * V3)
    return (delta * Y / (D * E) * V2 - delta * X / (C * E) * V3,
            X / (D * E) * V2 + Y / (C * E) * V3)


def velocity_from_uv(block_id, X, Y, U, V):
    """contravariant panel velocity (v2, v3) of an eastward / northward wind
    (U, V): CubedSphere::GetVyVz (cubed_sphere.cpp:138-151)"""
    return vec_abp_from_rll(X, Y, block_id, -U, V)


def uv_from_velocity(block_id, X, Y, v2, v3):
    """(U, V) of a contravariant panel velocity: CubedSphere::GetUV"""
    U, V = vec_rll_from_abp(X, Y, block_id, v2, v3)
    return -U, V
