"""Test systems.

``reference_test_systems`` rebuilds, as data, the systems that the reference
plugin's own test suite sets up in
platforms/reference/tests/TestReferenceTholeDipoleForce.cpp (two ammonia
molecules :62-199, four waters :318-430, the eight-water triclinic box
:562-641, the ZBisect ion + water :643-711, the ZOnly/Bisector triple :713-737
and the two-charge plasma system :761-780).  The reference asserts no numbers
for them (its expected values are placeholders), so they serve here as
input shapes: axis types, covalent maps, boxes and solver settings exactly as
those tests configure them.
"""
import numpy as np

from tholedipoleplugin_b200 import systems as S


def _system(pos, q, dip, pol, th, axis, cov12, cov13, **kw):
    n = len(q)
    kw.setdefault("masses", np.ones(n))
    return S.TholeSystem(positions=np.array(pos, dtype=np.float64), charges=np.array(q, dtype=np.float64),
                         dipoles=np.array(dip, dtype=np.float64), polarizabilities=np.array(pol, dtype=np.float64),
                         tholes=np.array(th, dtype=np.float64), axis=np.array(axis, dtype=np.int32),
                         cov12=[list(c) for c in cov12], cov13=[list(c) for c in cov13], **kw)


def ammonia(polarization=S.MUTUAL, method=S.NO_CUTOFF, scaled=False):
    n_dip = [8.3832254e-3, 0.0, 3.4232474e-3]
    h_dip = [-1.7388763e-3, 0.0, -4.6837475e-3]
    q = [-5.796e-1, 1.932e-1, 1.932e-1, 1.932e-1] * 2
    pol = [1.073e-3, 4.96e-4, 4.96e-4, 4.96e-4] * 2
    th = [3.9e-1] * 8
    dip = [n_dip, h_dip, h_dip, h_dip] * 2
    axis = [[2, 1, 2, 3], [2, 0, 2, 3], [2, 0, 1, 3], [2, 0, 1, 2],
            [2, 5, 6, 7], [2, 4, 6, 7], [2, 4, 5, 7], [2, 4, 5, 6]]
    cov12 = [[1, 2, 3], [0], [0], [0], [5, 6, 7], [4], [4], [4]]
    cov13 = [[], [2, 3], [1, 3], [1, 2], [], [6, 7], [5, 7], [5, 6]]
    pos = [[1.5927280e-01, 1.7000000e-06, 1.6491000e-03], [2.0805540e-01, -8.1258800e-02, 3.7282500e-02],
           [2.0843610e-01, 8.0953200e-02, 3.7462200e-02], [1.7280780e-01, 2.0730000e-04, -9.8741700e-02],
           [-1.6743680e-01, 1.5900000e-05, -6.6149000e-03], [-2.0428260e-01, 8.1071500e-02, 4.1343900e-02],
           [-6.7308300e-02, 1.2800000e-05, 1.0623300e-02], [-2.0426290e-01, -8.1231400e-02, 4.1033500e-02]]
    if scaled:  # the parameter change of testTholeDipoleAmmoniaMutualPolarization (:263-271)
        dip = [[d[0] * 0.7, d[1], d[2]] for d in dip]
        q = [1.1 * x for x in q]
        pol = [1.5 * x for x in pol]
        th = [1.3 * x for x in th]
    masses = [1.4007e1, 1.008, 1.008, 1.008] * 2
    return _system(pos, q, dip, pol, th, axis, cov12, cov13, method=method, box=np.array([0.6] * 3),
                   cutoff=9000000.0, polarization=polarization, target_eps=1e-6, max_iter=500,
                   masses=np.array(masses))


def water4(polarization=S.MUTUAL):
    o_dip = [0.0, 0.0, 7.5561214e-3]
    h_dip = [-2.0420949e-3, 0.0, -3.0787530e-3]
    q, pol, th, dip, axis, cov12, cov13 = [], [], [], [], [], [], []
    for jj in range(0, 12, 3):
        q += [-5.1966e-1, 2.5983e-1, 2.5983e-1]
        pol += [8.37e-4, 4.96e-4, 4.96e-4]
        th += [3.9e-1] * 3
        dip += [o_dip, h_dip, h_dip]
        axis += [[1, jj + 1, jj + 2, -1], [0, jj, jj + 2, -1], [0, jj, jj + 1, -1]]
        cov12 += [[jj + 1, jj + 2], [jj], [jj]]
        cov13 += [[], [jj + 2], [jj + 1]]
    pos = [[-8.7387270e-01, 5.3220410e-01, 7.4214000e-03], [-9.6050090e-01, 5.1173410e-01, -2.2202700e-02],
           [-8.5985900e-01, 4.9658230e-01, 1.0283390e-01], [9.1767100e-02, -7.8956650e-01, 4.3804200e-01],
           [1.2333420e-01, -7.0267430e-01, 4.2611550e-01], [1.7267090e-01, -8.2320810e-01, 4.8124750e-01],
           [8.6290110e-01, 6.2153500e-02, 4.1280850e-01], [8.6385200e-01, 1.2684730e-01, 3.3887060e-01],
           [9.5063550e-01, 5.3173300e-02, 4.4799160e-01], [5.0844930e-01, 2.8684740e-01, -6.9293750e-01],
           [6.0459330e-01, 3.0620510e-01, -7.0100130e-01], [5.0590640e-01, 1.8880920e-01, -6.8813470e-01]]
    masses = [1.5995e1, 1.008, 1.008] * 4
    return _system(pos, q, dip, pol, th, axis, cov12, cov13, method=S.PME, box=np.array([1.8643] * 3),
                   cutoff=0.7, polarization=polarization, target_eps=1e-6, max_iter=500, masses=np.array(masses))


def triclinic8():
    q = [-0.42616, 0.21308, 0.21308] * 8
    o_dip, h_dip = [0, 0, 0.0033078867454609203], [-0.0053536858428776405, 0, -0.014378273997907321]
    dip = [o_dip, h_dip, h_dip] * 8
    pol = [0.001 * 0.92, 0.001 * 0.539, 0.001 * 0.539] * 8
    th = [0.39] * 24
    axis, cov12, cov13 = [], [], []
    for i in range(8):
        a1, a2, a3 = 3 * i, 3 * i + 1, 3 * i + 2
        axis += [[1, a2, a3, -1], [0, a1, a3, -1], [0, a1, a2, -1]]
        cov12 += [[a2, a3], [a1], [a1]]
        cov13 += [[], [a3], [a2]]
    pos = [[0.867966, 0.708769, -0.0696862], [0.780946, 0.675579, -0.0382259], [0.872223, 0.681424, -0.161756],
           [-0.0117313, 0.824445, 0.683762], [0.0216892, 0.789544, 0.605003], [0.0444268, 0.782601, 0.75302],
           [0.837906, -0.0092611, 0.681463], [0.934042, 0.0098069, 0.673406], [0.793962, 0.0573676, 0.626984],
           [0.658995, 0.184432, -0.692317], [0.588543, 0.240231, -0.671793], [0.618153, 0.106275, -0.727368],
           [0.71466, 0.575358, 0.233152], [0.636812, 0.612604, 0.286268], [0.702502, 0.629465, 0.15182],
           [-0.242658, -0.850419, -0.250483], [-0.169206, -0.836825, -0.305829], [-0.279321, -0.760247, -0.24031],
           [-0.803838, -0.360559, 0.230369], [-0.811375, -0.424813, 0.301849], [-0.761939, -0.2863, 0.270962],
           [-0.148063, 0.824409, -0.827221], [-0.20902, 0.868798, -0.7677], [-0.0700878, 0.882333, -0.832221]]
    # Only the box diagonal enters the reference's minimum image (RTDF.cpp:1414-1423).
    box = np.array([1.8643, 1.8572057756524414, 1.8512735025730875])
    return _system(pos, q, dip, pol, th, axis, cov12, cov13, method=S.PME, box=box, cutoff=0.7,
                   polarization=S.MUTUAL, target_eps=1e-6, max_iter=60)


def zbisect():
    q = [-1.01875, 0, 0, 0, -0.51966, 0.25983, 0.25983]
    dip = [[0.06620218576365969, 0.056934176095985306, 0.06298584667720743], [0, 0, 0], [0, 0, 0], [0, 0, 0],
           [0, 0, 0.007556121391156931], [-0.05495981592297553, 0, -0.0030787530116780605],
           [-0.05495981592297553, 0, -0.0030787530116780605]]
    axis = [[2, 2, 1, 3], [5, -1, -1, -1], [5, -1, -1, -1], [5, -1, -1, -1], [1, 5, 6, -1], [0, 4, 6, -1],
            [0, 4, 5, -1]]
    pol = [0.001334, 0.001334, 0.001334, 0.001334, 0.000837, 0.000496, 0.000496]
    th = [0.39] * 7
    cov12, cov13 = [], []
    for i in range(4):
        cov12.append([0] if i != 0 else [])
        cov13.append([k for k in (1, 2, 3) if k != i])
    for i in range(4, 7):
        cov12.append([4] if i != 4 else [])
        cov13.append([k for k in (5, 6) if k != i])
    pos = [[-0.06317711175870899, -0.04905009196658128, 0.0767217],
           [-0.049166918626451395, -0.20747614470348363, 0.03979849999999996],
           [-0.19317150000000005, -0.05811762921948427, 0.1632788999999999],
           [0.04465103038516016, -0.018345116763806235, 0.18531239999999993],
           [0.005630299999999998, 0.40965770000000035, 0.5731495],
           [0.036148100000000016, 0.3627041999999996, 0.49299430000000033],
           [0.07781149999999992, 0.4178183000000004, 0.6355703000000004]]
    return _system(pos, q, dip, pol, th, axis, cov12, cov13, method=S.PME, box=np.array([4.0] * 3), cutoff=1.2,
                   polarization=S.MUTUAL, target_eps=1e-5, max_iter=60)


def zonly():
    d = [0.05, -0.05, 0.1]
    axis = [[S.ZONLY, 1, 0, 0], [S.BISECTOR, 0, 2, 0], [S.ZONLY, 1, 0, 0]]
    pos = [[0, 0, 0], [0.2, 0, 0], [0.2, 0.2, -0.05]]
    return _system(pos, [0.0] * 3, [d] * 3, [0.001] * 3, [0.39] * 3, axis, [[]] * 3, [[]] * 3,
                   method=S.NO_CUTOFF, polarization=S.MUTUAL, target_eps=1e-5, max_iter=60)


def plasma(charge0=1.0):
    pos = [[0.0, 0.0, 0.0], [0.3, 0.4, 0.0]]
    axis = [[S.NOAXISTYPE, 0, 0, 0]] * 2
    return _system(pos, [charge0, 1.0], [[0.0] * 3] * 2, [0.001] * 2, [0.39] * 2, axis, [[]] * 2, [[]] * 2,
                   method=S.PME, box=np.array([2.0] * 3), cutoff=1.0, polarization=S.MUTUAL, target_eps=1e-5,
                   max_iter=60)


def reference_test_systems():
    return [
        ("ammonia_direct", ammonia(S.DIRECT)),
        ("ammonia_mutual", ammonia(S.MUTUAL)),
        ("ammonia_extrapolated", ammonia(S.EXTRAPOLATED)),
        ("ammonia_scaled", ammonia(S.MUTUAL, scaled=True)),
        ("water4_pme", water4(S.MUTUAL)),
        ("water4_pme_direct", water4(S.DIRECT)),
        ("triclinic8", triclinic8()),
        ("zbisect", zbisect()),
        ("zonly", zonly()),
        ("plasma", plasma()),
    ]


def small_random_system(n, seed=0, method=S.NO_CUTOFF, polarization=S.MUTUAL, box=2.5, zonly_without_x=False):
    """Random mixed-axis-type system (threefold, z-bisect, bisector, z-then-x,
    z-only, no-axis) with ragged covalent lists, for stage-level checks.

    ZOnly atoms get an X atom unless ``zonly_without_x``: with X = -1 the
    reference's torque mapping indexes particleData[-1] (RTDF.cpp:1107,
    undefined), so such systems are only compared against the restatement's
    documented choice, never against the compiled reference."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, box, size=(n, 3))
    q = rng.normal(scale=0.4, size=n)
    dip = rng.normal(scale=0.01, size=(n, 3))
    pol = rng.uniform(0.3e-3, 1.5e-3, size=n)
    th = rng.uniform(0.3, 0.45, size=n)
    axis = np.full((n, 4), -1, dtype=np.int32)
    cov12, cov13 = [[] for _ in range(n)], [[] for _ in range(n)]
    for i in range(n):
        t = int(rng.integers(0, 6))
        others = [j for j in rng.permutation(n)[:4] if j != i][:3]
        axis[i, 0] = t
        if t != S.NOAXISTYPE:
            axis[i, 1] = others[0]
            if t != S.ZONLY or not zonly_without_x:
                axis[i, 2] = others[1]
            if t in (S.ZBISECT, S.THREEFOLD):
                axis[i, 3] = others[2]
        if t == S.ZTHENX and rng.random() < 0.5:
            axis[i, 3] = others[2]  # chiral check active
        k12 = int(rng.integers(0, 4))
        cov12[i] = [int(j) for j in rng.integers(0, n, size=k12)]
        k13 = int(rng.integers(0, 4))
        cov13[i] = [int(j) for j in rng.integers(0, n, size=k13)]
    return S.TholeSystem(positions=pos, charges=q, dipoles=dip, polarizabilities=pol, tholes=th, axis=axis,
                         cov12=cov12, cov13=cov13, method=method, box=np.array([box] * 3), cutoff=0.5 * box * 0.9,
                         polarization=polarization, target_eps=1e-8, max_iter=300, masses=rng.uniform(1, 16, n))


def sparse_clumps(n_clumps=12, waters_per_clump=11, box=10.0, seed=21, polarization=S.MUTUAL):
    """Compact clumps of waters scattered through a large periodic box, stored
    clump by clump.  Each 32-atom tile is then spatially small while tiles sit
    up to a box diagonal apart, which exercises both the tile-level minimum
    image (no per-pair folding) and per-pair folding near the half box."""
    rng = np.random.default_rng(seed)
    centres = []
    for _ in range(n_clumps):
        c = rng.uniform(0, box, size=3)
        k = 3
        g = (np.arange(k) - 1) * 0.31
        gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
        sites = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)[:waters_per_clump]
        centres.append(c + sites + rng.uniform(-0.02, 0.02, size=sites.shape))
    centres = np.concatenate(centres)
    pos = S.place_waters(centres, rng)
    nw = centres.shape[0]
    charges, dip, pol, th, axis, cov12, cov13, masses = S._water_parameters(nw)
    return S.TholeSystem(positions=pos, charges=charges, dipoles=dip, polarizabilities=pol, tholes=th, axis=axis,
                         cov12=cov12, cov13=cov13, method=S.PME, box=np.array([box] * 3), cutoff=0.9,
                         polarization=polarization, target_eps=1e-6, max_iter=500, masses=masses)
