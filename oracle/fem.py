"""CPU oracle (test infrastructure only) for the finite-element pair weights of P1 triangles
(src/warpSPHBoundaries/edge/warpbc.py:226-345, 486-510).  Only tests/ use this module, as the checker.

Per (query, triangle) pair: the triangle's channels as a polygon from oracle/edge2d.local_twelve (the reference's
closed-form edge channels and indicator, pinned to its 40-digit golden vectors), combined with the barycentric
functions phi_k(x + h y) = l_k + g_k . y of the element's own vertex order:
    w_k = l_k lam + g_k . m1 / h          G_kj = l_k G_j + sum_d g_kd g1_dj / h      (physical units)
No far-field rule: the oracle is the exact integral everywhere."""
import numpy as np

from oracle import edge2d as O


def pair_weights(pair_q, pair_e, positions, supports, vertices, elements, kernel):
    pos = np.asarray(positions, float).reshape(-1, 2)
    sup = np.asarray(supports, float).reshape(-1)
    V = np.asarray(vertices, float).reshape(-1, 2)
    E = np.asarray(elements, np.int64).reshape(-1, 3)
    P = len(pair_q)
    w = np.zeros((P, 3))
    G = np.zeros((P, 3, 2))
    for k, (q, e) in enumerate(zip(np.asarray(pair_q), np.asarray(pair_e))):
        h, x = sup[q], pos[q]
        T = V[E[e]]
        r = (T - x) / h
        d2 = (r[1, 0] - r[0, 0]) * (r[2, 1] - r[0, 1]) - (r[1, 1] - r[0, 1]) * (r[2, 0] - r[0, 0])
        l, g = np.zeros(3), np.zeros((3, 2))
        for i in range(3):
            a, b = r[(i + 1) % 3], r[(i + 2) % 3]
            l[i] = (a[0] * b[1] - a[1] * b[0]) / d2
            g[i] = [(a[1] - b[1]) / d2, (b[0] - a[0]) / d2]
        ccw = T if d2 > 0 else T[[0, 2, 1]]
        ch = O.local_twelve(ccw, np.array([[0, 1], [1, 2], [2, 0]]), 0, x[None], np.array([h]), kernel, h)[0]
        lam, m1, Gc, g1 = ch[0], ch[1:3], ch[3:5], ch[5:9].reshape(2, 2)
        for i in range(3):
            w[k, i] = l[i] * lam + g[i] @ m1 / h
            G[k, i] = l[i] * Gc + g[i] @ g1 / h
    return w, G
