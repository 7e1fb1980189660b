"""Triangulated surfaces (numpy) for the triangle FMM: icospheres and a two-body mesh, used by
the tests and the bench as synthetic inputs."""
import numpy as np


def icosphere(k, radius=1.0, center=(0.0, 0.0, 0.0), axes=(1.0, 1.0, 1.0)):
    """Icosahedron subdivided k times onto the unit sphere (20 * 4^k triangles, vertices ordered
    so that (v2 - v1) x (v3 - v1) points outward), scaled per axis, by radius, then shifted.
    Returns (N, 3, 3) vertex coordinates."""
    t = (1 + 5 ** 0.5) / 2
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    V /= np.linalg.norm(V, axis=1)[:, None]
    for _ in range(k):
        # one midpoint per edge: edges keyed by their sorted vertex pair
        E = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.sort(E, axis=1)
        uniq, inv = np.unique(key[:, 0].astype(np.int64) * len(V) + key[:, 1], return_inverse=True)
        a, b = uniq // len(V), uniq % len(V)
        M = (V[a] + V[b]) / 2
        M /= np.linalg.norm(M, axis=1)[:, None]
        mid = len(V) + inv.reshape(3, -1)          # midpoints of edges (0,1), (1,2), (2,0) of every face
        ab, bc, ca = mid[0], mid[1], mid[2]
        F = np.concatenate([np.stack([F[:, 0], ab, ca], 1), np.stack([F[:, 1], bc, ab], 1),
                            np.stack([F[:, 2], ca, bc], 1), np.stack([ab, bc, ca], 1)])
        V = np.concatenate([V, M])
    T = V[F] * np.asarray(axes, float) * radius + np.asarray(center, float)
    # outward orientation
    n = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    flip = np.einsum("ij,ij->i", n, T.mean(axis=1) - np.asarray(center, float)) < 0
    T[flip] = T[flip][:, [0, 2, 1]]
    return T


def normals_centroids(T):
    n = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    return n / np.linalg.norm(n, axis=1)[:, None], T.mean(axis=1)


def two_spheres(k_big=4, k_small=5):
    """A coarse unit sphere and a finely meshed small ellipsoid beside it: uneven triangle
    sizes, so the tree is adaptive (lists 3 and 4 are not empty)."""
    return np.concatenate([icosphere(k_big), icosphere(k_small, 0.15, (1.4, 0.2, 0.1), (1.0, 0.7, 0.5))])
