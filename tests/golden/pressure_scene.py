"""The lattice and initial state of oracle/ref/harness_step.c in its pressure
mode, rebuilt here so that the pressure-inlet fixture needs to keep only the
reference's results: a tube of radius 4 along k (centre i = 20, j = 30,
1-based) with a phase-5 ball, fluid for 6 < k < 20, the end layers k = 6 and
k = 20 pressure inlet/outlet points of two codes, walls at every non-fluid
point linked to the tube; populations w_c (1 + 0.02 (u - 1/2)) and a body
force 2e-3 (u - 1/2) (+1e-3 along k) from the harness's xorshift generator.

Arrays are in a 0-based box of 13 x 13 x 17 points whose corner is the
reference's (14, 24, 5)."""
import numpy as np

CI, CJ, TUBE_R2, K_LO, K_HI = 20, 30, 16, 6, 20
BOX_LO = (CI - 6, CJ - 6, K_LO - 1)  # 1-based reference indices of box[0, 0, 0]
SHAPE = (13, 13, K_HI - K_LO + 3)
STEPS = 5
E = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [-1, -1, 0],
              [-1, 1, 0], [1, -1, 0], [1, 0, 1], [-1, 0, -1], [-1, 0, 1], [1, 0, -1], [0, 1, 1], [0, -1, -1],
              [0, -1, 1], [0, 1, -1]])


def lattice(code_lo, code_hi):
    b = -np.ones(SHAPE, np.int32)
    for ii in range(SHAPE[0]):
        for jj in range(SHAPE[1]):
            for kk in range(SHAPE[2]):
                i, j, k = ii + BOX_LO[0], jj + BOX_LO[1], kk + BOX_LO[2]
                r2 = (i - CI) ** 2 + (j - CJ) ** 2
                b2 = r2 + (k - 13) ** 2
                if r2 < TUBE_R2 and K_LO < k < K_HI:
                    b[ii, jj, kk] = 5 if b2 < 5 else 1
                if r2 < TUBE_R2 and k == K_LO:
                    b[ii, jj, kk] = code_lo
                if r2 < TUBE_R2 and k == K_HI:
                    b[ii, jj, kk] = code_hi
    marked = b.copy()
    for ii, jj, kk in np.argwhere(b <= 0):
        for e in E:
            p = (ii + e[0], jj + e[1], kk + e[2])
            if all(0 <= p[a] < SHAPE[a] for a in range(3)) and b[p] > 0:
                marked[ii, jj, kk] = 0
                break
    return marked


def initial_state(n):
    """Populations [19][n] and body force [3][n] as the harness draws them."""
    mask = (1 << 64) - 1
    st = [0x9E3779B97F4A7C15]

    def u01():
        r = st[0]
        r ^= (r << 13) & mask
        r ^= r >> 7
        r ^= (r << 17) & mask
        st[0] = r
        return (r >> 11) * (1.0 / 9007199254740992.0)
    w = [np.float32(1 / 18)] * 6 + [np.float32(1 / 36)] * 12 + [np.float32(1 / 3)]
    f = np.empty((19, n), np.float32)
    bf = np.empty((3, n), np.float32)
    for l in range(n):
        for c in range(19):
            f[c, l] = np.float32(float(w[c]) * (1.0 + 0.02 * (u01() - 0.5)))
        for a in range(3):
            bf[a, l] = np.float32(2e-3 * (u01() - 0.5) + (1e-3 if a == 2 else 0.0))
    return f, bf


# the five runs of the fixture: (inlet code at k = 6, code at k = 20, the
# iteration before the first step); together they cover the nine waveforms
# and both branches of each kind
RUNS = ((1001, 1003, 100000), (1002, 1004, 300000), (1005, 1006, 200000), (1007, 1008, 500000),
        (1009, 1001, 650000))
