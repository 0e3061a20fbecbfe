"""Regenerates tests/golden/ref_*.npz from the reference's own regression
fixtures (test infrastructure; run in a container where the reference tree
is mounted, e.g. ``python tests/golden/make_reference_fixtures.py
/path/to/dust``).

The reference stores, for each regression case, the solver's state at output
step 11 in an HDF5 file (tests/sym_test/static/<case>/Output/ref_res_0011.h5,
written by save_status, src/io/mod_dust_io.f90:127-437).  save_status runs
after solve_linsys (src/dust.f90:648) and before update_wake (:1071), so the
panel wake (PanelWake/WakePoints, StartPoints, WakeVort), the end vortices
(the last wake row's far edge with ParticleWake/LastPanIdou) and the
particles (ParticleWake/WakePoints, WakeVort) in the file are exactly the
wake that step's linear system was assembled against, and
Components/*/Solution/Vort is its solution.

The body geometry is not in the file (output_detailed_geo = F), so it is
rebuilt here from the case's parametric input the way the reference's
pre-processor builds it:

* read_mesh_parametric (src/io/mod_parametric_io.f90:83-895): connectivity,
  chordwise division (define_division :1300-1333), sections from the NACA
  4-digit mean line for vortex-lattice elements (define_section :899-969,
  naca4digits :973-1055), regions by uniform spanwise interpolation with
  sweep and dihedral offsets;
* symmetry_mesh_structured (src/geo/mod_build_geo.f90:1359-1532): the
  reflected half, sewn at the root section, elements re-ordered;
* the component's reference frame (References.in): x_global = R x + origin.

The rebuilt trailing-edge nodes must coincide with the first row of the
saved panel-wake points (they are its start points, mod_wake.f90:485-487),
which this script checks to 1e-12 before writing.

Each fixture (.npz) holds: the body panels ``ver`` (n, 4, 3); the wake
panels ``wake_ver`` (implicit first row, then the explicit rows) with
``wake_mag``; ``impl_ind`` (1-based generating elements of the implicit
row); the end vortices ``end_ver``/``end_mag``; the particles ``part_cen``,
``part_alpha`` (circulation vector mag * dir) and ``part_rv``; the
parameters; and ``vort_ref``, the reference's solved doublet intensities.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import h5v0  # noqa: E402


# ----------------------------------------------------------- input files
def parse_in(path):
    """key = value lines of a DUST input file ('!' comments, Fortran array
    constructors (/ ... /)); repeated keys keep every value in order.
    Blocks in braces (motion = {...}) are skipped."""
    out = {}
    depth = 0
    for raw in open(path):
        line = raw.split("!")[0].strip()
        if not line:
            continue
        if "{" in line:
            depth += line.count("{")
        if depth > 0:
            depth -= line.count("}")
            continue
        if "=" not in line:
            continue
        k, v = (s.strip() for s in line.split("=", 1))
        out.setdefault(k.lower(), []).append(v)
    return out


def as_float(v):
    return float(v.replace("d", "e").replace("D", "e"))


def as_vec(v):
    m = re.match(r"\(/(.*)/\)", v.strip())
    return np.array([as_float(x) for x in m.group(1).split(",")])


def as_bool(v):
    return v.strip().upper().startswith("T")


# --------------------------------------------------- parametric geometry
def define_division(kind, nelem):
    """define_division (mod_parametric_io.f90:1300-1333)."""
    step = 1.0 / (float(nelem) + 1e-12)
    i = np.arange(nelem + 1, dtype=np.float64)
    if kind == "uniform":
        return i * step
    if kind == "cosine":
        return (1.0 - np.cos(np.pi * i * step)) / 2.0
    if kind in ("cosineLE", "cosineIB"):
        return 1.0 - np.cos(np.pi / 2.0 * i * step)
    if kind in ("cosineTE", "cosineOB"):
        return np.sin(np.pi / 2.0 * (i * step))
    raise ValueError(kind)


def naca4(name, xa):
    """naca4digits (mod_parametric_io.f90:973-1055): mean line and the
    closed-TE surface points (lower reversed, then upper)."""
    m = int(name[0]) / 100.0
    p = int(name[1]) / 10.0
    s = int(name[2:4]) / 100.0
    ml = np.zeros_like(xa)
    th = np.zeros_like(xa)
    if p > 0:
        a = xa <= p
        ml[a] = m / p ** 2 * (2.0 * p * xa[a] - xa[a] ** 2)
        th[a] = 2.0 * m / p ** 2 * (p - xa[a])
        b = ~a
        ml[b] = m / (1.0 - p) ** 2 * (1.0 - 2.0 * p + 2.0 * p * xa[b] - xa[b] ** 2)
        th[b] = 2.0 * m / (1.0 - p) ** 2 * (p - xa[b])
    t = 5.0 * s * (0.2969 * np.sqrt(xa) - 0.1260 * xa - 0.3516 * xa ** 2 + 0.2843 * xa ** 3
                   - 0.1036 * xa ** 4)
    mean = np.stack([xa, ml])
    up = np.stack([xa - t * np.sin(th), ml + t * np.cos(th)])
    lo = np.stack([xa + t * np.sin(th), ml - t * np.cos(th)])
    n = len(xa) - 1
    pts = np.concatenate([lo[:, n:0:-1], up], axis=1)
    return mean, pts


def define_section(chord, airfoil, twist, eltype, division, ref_frac):
    """define_section (mod_parametric_io.f90:899-969) for NACA 4-digit
    airfoils: (2, npoints) section points, twisted about the reference
    chord fraction."""
    if not (airfoil.upper().startswith("NACA") and len(airfoil) == 8):
        raise ValueError("only NACA 4-digit sections are restated here: " + airfoil)
    mean, pts = naca4(airfoil[4:8], division)
    pl = (mean if eltype == "v" else pts).copy()
    pl[0] = pl[0] - ref_frac
    pl = pl * chord
    tw = twist * 4.0 * np.arctan(1.0) / 180.0
    # matmul(reshape((/cos, -sin, sin, cos/), (/2,2/)), pl): column-major 2x2
    M = np.array([[np.cos(tw), np.sin(tw)], [-np.sin(tw), np.cos(tw)]])
    return M @ pl


def read_mesh_parametric(inp):
    """read_mesh_parametric (mod_parametric_io.f90:83-895) without hinges
    and with the default constant twist per region.  Returns (ee, rr,
    npoints_chord, nelem_span): ee (4, ne) 1-based, rr (3, np)."""
    eltype = inp["el_type"][0].strip()
    nelem_chord = int(inp["nelem_chord"][0])
    type_chord = inp.get("type_chord", ["uniform"])[0].split()[0]
    ref_point = as_vec(inp.get("starting_point", ["(/0.0, 0.0, 0.0/)"])[0])
    ref_frac = as_float(inp.get("reference_chord_fraction", ["0.0"])[0])
    chords = [as_float(v) for v in inp["chord"]]
    twists = [as_float(v) for v in inp["twist"]]
    airfoils = [v.split()[0] for v in inp["airfoil"]]
    spans = [as_float(v) for v in inp["span"]]
    sweeps = [as_float(v) for v in inp["sweep"]]
    diheds = [as_float(v) for v in inp["dihed"]]
    nspan = [int(v) for v in inp["nelem_span"]]
    tspan = [v.split()[0] for v in inp.get("type_span", ["uniform"] * len(spans))]
    assert len(chords) == len(spans) + 1
    nct = 2 * nelem_chord if eltype == "p" else nelem_chord
    npc = nct + 1
    nst = sum(nspan)
    ee = np.zeros((4, nct * nst), dtype=np.int64)
    for ic in range(1, nct + 1):
        for isp in range(1, nst + 1):
            ie = nct * (isp - 1) + ic
            ip = npc * (isp - 1) + ic
            ee[:, ie - 1] = [ip + npc, ip, ip + 1, ip + npc + 1]
    rr = np.zeros((3, npc * (nst + 1)))
    division = define_division(type_chord, nelem_chord)
    dx, dy, dz = ref_point
    ista, iend = 0, npc
    sec2 = None
    for ir in range(len(spans)):
        if ir == 0:
            xy1 = define_section(chords[0], airfoils[0], twists[0], eltype, division, ref_frac)
            sec1 = np.stack([xy1[0] + ref_point[0], np.zeros(npc) + ref_point[1],
                             xy1[1] + ref_point[2]])
            rr[:, ista:iend] = sec1
        else:
            sec1 = sec2
        xy2 = define_section(chords[ir + 1], airfoils[ir + 1], twists[ir + 1], eltype,
                             division, ref_frac)
        dx = spans[ir] * np.tan(sweeps[ir] * np.pi / 180.0) + dx
        dy = spans[ir] + dy
        dz = spans[ir] * np.tan(diheds[ir] * np.pi / 180.0) + dz
        sec2 = np.stack([xy2[0] + dx, np.zeros(npc) + dy, xy2[1] + dz])
        for i1 in range(1, nspan[ir] + 1):
            ista, iend = iend, iend + npc
            if tspan[ir] == "uniform":
                rr[:, ista:iend] = sec1 + float(i1) / float(nspan[ir]) * (sec2 - sec1)
            else:
                raise ValueError("only uniform spanwise division is restated here")
    return ee, rr, npc, nst


def symmetry_mesh_structured(ee, rr, npc, nelems_span, cent, norm, eps=1e-2):
    """symmetry_mesh_structured (mod_build_geo.f90:1359-1532), for a
    component whose first (root) section lies on the symmetry plane."""
    d_all = (rr - cent[:, None]).T @ norm
    on = np.abs(d_all) < eps
    assert on[0] and not on[-1] and on.sum() == npc, "root section must be sewn"
    ne, np_ = ee.shape[1], rr.shape[1]
    et = np.zeros((4, 2 * ne), dtype=np.int64)
    et[:, :ne] = ee
    for ie in range(ne):
        et[0, ne + ie] = np_ - npc + ee[1, ie]
        et[1, ne + ie] = np_ - npc + ee[0, ie]
        et[2, ne + ie] = np_ - npc + ee[3, ie]
        et[3, ne + ie] = np_ - npc + ee[2, ie]
    et[0, ne:ne + npc - 1] = np.arange(1, npc)
    et[3, ne:ne + npc - 1] = np.arange(2, npc + 1)
    n = norm / np.linalg.norm(norm)
    l = float(np.dot(cent, n))
    rt = np.zeros((3, 2 * np_ - npc))
    rt[:, :np_] = rr
    for ip in range(1, np_ - npc + 1):
        d = float(np.dot(rr[:, ip + npc - 1], n)) - l
        rt[:, np_ + ip - 1] = rt[:, npc + ip - 1] - 2 * d * n
    nec = npc - 1
    es = np.zeros_like(et)
    for i1 in range(1, nelems_span + 1):
        es[:, (i1 - 1) * nec:i1 * nec] = et[:, 2 * ne - i1 * nec:2 * ne - (i1 - 1) * nec]
    for i1 in range(1, nelems_span + 1):
        es[:, (i1 - 1) * nec + ne:i1 * nec + ne] = et[:, (i1 - 1) * nec:i1 * nec]
    return es, rt


def reference_frame(refs_in, tag):
    """(R, origin) of reference `tag` from a References.in (static frames
    with parent 0)."""
    blocks = open(refs_in).read().split("reference_tag")
    for blk in blocks[1:]:
        p = parse_in_text("reference_tag" + blk)
        if p["reference_tag"][0].strip() == tag:
            assert p.get("parent_tag", ["0"])[0].strip() == "0"
            org = as_vec(p["origin"][0])
            R = as_vec(p["orientation"][0]).reshape(3, 3).T  # Fortran column order
            return R, org
    raise KeyError(tag)


def parse_in_text(text):
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as fh:
        fh.write(text)
        name = fh.name
    try:
        return parse_in(name)
    finally:
        os.unlink(name)


# ------------------------------------------------------------- the case
def build_case(case_dir):
    pre = parse_in(os.path.join(case_dir, "dust_pre.in"))
    assert len(pre["comp_name"]) == 1, "one component per case here"
    geo = parse_in(os.path.join(case_dir, pre["geo_file"][0].strip()))
    ref_tag = pre["ref_tag"][0].strip()
    ee, rr, npc, nst = read_mesh_parametric(geo)
    if as_bool(geo.get("mesh_symmetry", ["F"])[0]):
        ee, rr = symmetry_mesh_structured(ee, rr, npc, nst,
                                          as_vec(geo["symmetry_point"][0]),
                                          as_vec(geo["symmetry_normal"][0]))
        nst = 2 * nst
    R, org = reference_frame(os.path.join(case_dir, "References.in"), ref_tag)
    rg = (R @ rr) + org[:, None]
    ver = np.transpose(rg[:, ee - 1], (2, 1, 0))  # (ne, 4, 3)
    return geo["el_type"][0].strip(), ver, npc - 1, nst


def extract(case_dir, name):
    eltype, ver, nch, nsp = build_case(case_dir)
    f = h5v0.File(os.path.join(case_dir, "Output", "ref_res_0011.h5"))
    at = f.attrs()
    comps = f["Components"]
    vort = np.concatenate([comps[k]["Solution/Vort"].read()
                           for k in sorted(comps.keys()) if k.startswith("Comp")])
    wp = f["PanelWake/WakePoints"].read()        # (rows+1, points, 3)
    sp = f["PanelWake/StartPoints"].read() - 1   # (stripes, 2), 0-based
    wv = f["PanelWake/WakeVort"].read()          # (rows, stripes)
    last = f["ParticleWake/LastPanIdou"].read()
    pc = f["ParticleWake/WakePoints"].read()
    pa = f["ParticleWake/WakeVort"].read()
    nrow = wv.shape[0]
    nstripe = sp.shape[0]
    assert nstripe == nsp
    # build_te_parametric (src/geo/mod_build_geo.f90:2227-2330): trailing
    # edge elements per spanwise strip i (1-based) are e_te(1) = i * nch and,
    # for surface panels, e_te(2) = 1 + (i - 1) * nch (the two sides of the
    # closed trailing edge); the trailing-edge nodes are the midpoints of
    # i_te(1:2, k), which are the wake's start points (mod_wake.f90:485-487)
    ee_ver = ver  # (ne, 4, 3): vertices in ee order
    i_strip = np.arange(1, nsp + 1)
    impl = np.zeros((nstripe, 2), dtype=np.int32)
    impl[:, 0] = i_strip * nch
    if eltype == "p":
        impl[:, 1] = 1 + (i_strip - 1) * nch
        te0 = 0.5 * (ee_ver[0, 1] + ee_ver[nch - 1, 2])
        te_rest = 0.5 * (ee_ver[(i_strip - 1) * nch, 0] + ee_ver[i_strip * nch - 1, 3])
    else:
        te0 = ee_ver[nch - 1, 2]
        te_rest = ee_ver[i_strip * nch - 1, 3]
    rr_te = np.concatenate([te0[None], te_rest])
    worst = float(np.abs(rr_te - wp[0]).max())
    assert worst < 1e-12, "rebuilt trailing edge differs from the wake start points by %g" % worst
    # ii_te: stripe i spans trailing-edge nodes (i + 1, i)
    assert np.array_equal(sp[:, 0], i_strip) and np.array_equal(sp[:, 1], i_strip - 1)
    wver = []
    for ir in range(nrow):
        for iw in range(nstripe):
            p1, p2 = sp[iw]
            wver.append([wp[ir, p1], wp[ir, p2], wp[ir + 1, p2], wp[ir + 1, p1]])
    wver = np.asarray(wver)
    wmag = np.concatenate([np.zeros(nstripe)] + [wv[ir] for ir in range(1, nrow)])
    end_ver = np.stack([wp[nrow, sp[:, 0]], wp[nrow, sp[:, 1]]], axis=1)
    rv = float(at["VortexRad"])
    try:
        prv = f["ParticleWake/VortexRad"].read()
    except KeyError:  # older writers: every particle has sim_param%VortexRad
        prv = np.full(len(pc), rv)
    out = dict(
        eltype=eltype, ver=ver, nver=np.full(len(ver), 4, dtype=np.int32),
        wake_ver=wver, wake_mag=wmag, impl_ind=impl, end_ver=end_ver, end_mag=last,
        part_cen=pc, part_alpha=pa, part_rv=prv,
        u_inf=np.asarray(at["u_inf"], dtype=np.float64), rankine_rad=float(at["RankineRad"]),
        vortex_rad=rv, cutoff_rad=float(at["CutoffRad"]),
        far_field_ratio_doublet=float(at["FarFieldRatioDoublet"]),
        vort_ref=vort, te_match=worst, time=float(f["time"].read()),
        source=name)
    return out


def extract_step_pair(case_dir, name):
    """Two consecutive result files (output steps 10 and 11, dt_out = dt) of a
    fmm = F vortex-lattice case: the state that step 10's update_wake and
    complete_wake start from (saved after solve_linsys, before update_wake)
    and the particles, panel wake and last intensities they produce, as
    saved at step 11 (src/dust.f90:648, 1017, 1071, 1108)."""
    eltype, ver, nch, nsp = build_case(case_dir)
    assert eltype == "v", "vortex-lattice trailing edge only"
    f10 = h5v0.File(os.path.join(case_dir, "Output", "ref_res_0010.h5"))
    f11 = h5v0.File(os.path.join(case_dir, "Output", "ref_res_0011.h5"))
    at = f10.attrs()

    def comp_vort(f):
        comps = f["Components"]
        return np.concatenate([comps[k]["Solution/Vort"].read()
                               for k in sorted(comps.keys()) if k.startswith("Comp")])

    sp = f10["PanelWake/StartPoints"].read()  # (stripes, 2), 1-based
    i_strip = np.arange(1, nsp + 1)
    assert np.array_equal(sp[:, 0], i_strip + 1) and np.array_equal(sp[:, 1], i_strip)
    # build_te_parametric (src/geo/mod_build_geo.f90:2244-2310), vortex
    # lattice: e_te(1, i) = i nch; neighbours i +- 1 with orientation 1, none
    # at the ends; t_te from the trailing element's side edges, normalised
    gen = np.zeros((nsp, 2), dtype=np.int32)
    gen[:, 0] = i_strip * nch
    neigh = np.stack([i_strip + 1, i_strip - 1], axis=1).astype(np.int32)
    neigh[-1, 0] = 0
    neigh[0, 1] = 0
    neigh_o = np.ones((nsp, 2), dtype=np.int32)
    neigh_o[-1, 0] = 0
    neigh_o[0, 1] = 0
    t_te = np.zeros((nsp + 1, 3))
    e1 = ver[gen[0, 0] - 1]
    t_te[0] = 0.5 * (e1[2] - e1[1])
    for i1 in range(1, nsp + 1):
        e = ver[gen[i1 - 1, 0] - 1]
        t_te[i1] = 0.5 * (e[3] - e[0])
    t_te = t_te / np.sqrt((t_te ** 2).sum(axis=1))[:, None]
    wp10 = f10["PanelWake/WakePoints"].read()
    te_pts = np.concatenate([ver[nch - 1, 2][None], ver[i_strip * nch - 1, 3]])
    worst = float(np.abs(te_pts - wp10[0]).max())
    assert worst < 1e-12, "rebuilt trailing edge differs from the wake start points by %g" % worst
    out = dict(
        eltype=eltype, ver=ver, nver=np.full(len(ver), 4, dtype=np.int32),
        ii=sp.astype(np.int32), neigh=neigh, neigh_o=neigh_o, gen=gen,
        te_pts=te_pts, te_dir=t_te, te_scaling=float(at["first_panel_scaling"]),
        vort10=comp_vort(f10),
        wake_pts10=wp10, wake_vel10=f10["PanelWake/WakeVels"].read(),
        wake_vort10=f10["PanelWake/WakeVort"].read(),
        last10=f10["ParticleWake/LastPanIdou"].read(),
        part_cen10=f10["ParticleWake/WakePoints"].read(),
        part_alpha10=f10["ParticleWake/WakeVort"].read(),
        part_rv10=f10["ParticleWake/VortexRad"].read(),
        part_vel10=f10["ParticleWake/WakeVels"].read(),
        wake_pts11=f11["PanelWake/WakePoints"].read(),
        wake_vort11=f11["PanelWake/WakeVort"].read(),
        last11=f11["ParticleWake/LastPanIdou"].read(),
        part_cen11=f11["ParticleWake/WakePoints"].read(),
        part_alpha11=f11["ParticleWake/WakeVort"].read(),
        part_rv11=f11["ParticleWake/VortexRad"].read(),
        u_inf=np.asarray(at["u_inf"], dtype=np.float64), u_ref=float(at["u_ref"]),
        dt=float(at["dt"]), box_min=np.asarray(at["particles_box_min"], dtype=np.float64),
        box_max=np.asarray(at["particles_box_max"], dtype=np.float64),
        n_wake_panels=int(at["n_wake_panels"]), n_wake_particles=int(at["n_wake_particles"]),
        min_vel_at_te=float(at["min_vel_at_te"]),
        rankine_rad=float(at["RankineRad"]), vortex_rad=float(at["VortexRad"]),
        k_vortex_rad=float(at["KVortexRad"]), cutoff_rad=float(at["CutoffRad"]),
        far_field_ratio_doublet=float(at["FarFieldRatioDoublet"]),
        nu_inf=float(at["mu_inf"]) / float(at["rho_inf"]),
        vortstretch=int(at["Vortstretch"] in (True, "T", 1)),
        diffusion=int(at["vortdiff"] in (True, "T", 1)),
        penetration_avoidance=int(at["PenetrationAvoidance"] in (True, "T", 1)),
        pa_check_radius=float(at["PenetrationAvoidanceCheckRadius"]),
        pa_element_radius=float(at["PenetrationAvoidanceElementRadius"]),
        te_match=worst, time10=float(f10["time"].read()), time11=float(f11["time"].read()),
        source=name)
    return out


CASES = {"sym_static_v": "tests/sym_test/static/v",
         "sym_static_p": "tests/sym_test/static/p"}
STEP_PAIRS = {"sym_static_nl_v_steps_10_11": "tests/sym_test/static/nl_v"}


DEFAULT_ROOT = os.environ.get("DUST_REFERENCE_ROOT", "/root/reference")


def main(ref_root, out_dir=HERE):
    for name, rel in CASES.items():
        d = extract(os.path.join(ref_root, rel), name)
        path = os.path.join(out_dir, "ref_%s.npz" % name)
        np.savez_compressed(path, **d)
        print("%s: %d elements, %d wake panels, %d particles, TE match %.1e -> %s"
              % (name, len(d["ver"]), len(d["wake_ver"]), len(d["part_cen"]), d["te_match"],
                 os.path.relpath(path)))
    for name, rel in STEP_PAIRS.items():
        d = extract_step_pair(os.path.join(ref_root, rel), name)
        path = os.path.join(out_dir, "ref_%s.npz" % name)
        np.savez_compressed(path, **d)
        print("%s: %d elements, %d -> %d particles, TE match %.1e -> %s"
              % (name, len(d["ver"]), len(d["part_cen10"]), len(d["part_cen11"]),
                 d["te_match"], os.path.relpath(path)))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_ROOT)
