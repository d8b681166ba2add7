"""Extract the known-answer values that pin the Delhommeau path from the
reference's own test suite and write them to ``reference_golden.json``.

Run in a checkout that has the reference next to it:

    python tests/golden/make_golden.py /path/to/capytaine

Sources (paths inside the capytaine project):
* pytest/test_consistency_with_Nemoh_2.py:61-99  - 6x6 S matrices at k=0 and
  k=inf on a hand-built 7-vertex mesh (8 significant digits).
* pytest/test_consistency_with_Nemoh_2.py:36-58  - immersed sphere added mass.
* pytest/test_consistency_with_Nemoh_2.py:101-153 - floating sphere at omega=1,2.
* pytest/test_consistency_with_Nemoh_2.py:155-172 - same sphere, rho=450, g=1.625.
* pytest/test_consistency_with_Nemoh_2.py:175-203 - same sphere in 10 m of water.
* pytest/test_consistency_with_Nemoh_2.py:206-226 - two spheres 20 m apart in 10 m of water.
* pytest/test_consistency_with_Nemoh_2.py:228-270 - submerged sphere and horizontal cylinder,
  4 x 4 added mass and damping (rows: influenced dofs, columns: radiating dofs).
The values are read from the test source with ``ast``; nothing is executed.
"""
import ast
import json
import os
import sys


def _literal(node):
    """Evaluate a literal expression possibly wrapped in np.array(...)/np.exp(...)."""
    if isinstance(node, ast.Call) and getattr(node.func, "attr", None) == "array":
        return ast.literal_eval(node.args[0])
    return ast.literal_eval(node)


def _complex_polar(node):
    """Parse ``A * np.exp(Bj)`` into [A, B] (modulus, phase in radians)."""
    assert isinstance(node, ast.BinOp) and isinstance(node.op, ast.Mult)
    mod = ast.literal_eval(node.left)
    call = node.right
    arg = call.args[0]
    if isinstance(arg, ast.UnaryOp):
        phase = -ast.literal_eval(arg.operand).imag
    else:
        phase = ast.literal_eval(arg).imag
    return [mod, phase]


def _isclose_calls(fn):
    out = []
    for node in ast.walk(fn):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", None) == "isclose":
            out.append(node)
    out.sort(key=lambda n: n.lineno)
    return out


def main(ref_root):
    path = os.path.join(ref_root, "pytest", "test_consistency_with_Nemoh_2.py")
    tree = ast.parse(open(path).read())
    funcs = {n.name: n for n in tree.body if isinstance(n, ast.FunctionDef)}
    golden = {"source": "pytest/test_consistency_with_Nemoh_2.py"}

    fn = funcs["test_build_matrix_of_rankine_and_reflected_rankine"]
    s_refs = []
    for node in ast.walk(fn):
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name in ("vertices", "faces"):
                golden[f"rankine_mesh_{name}"] = _literal(node.value)
            elif name == "S_ref":
                s_refs.append((node.lineno, _literal(node.value)))
    s_refs.sort()
    golden["S_k0"] = s_refs[0][1]
    golden["S_kinf"] = s_refs[1][1]

    fn = funcs["test_immersed_sphere"]
    vals = [ast.literal_eval(c.args[1]) for c in _isclose_calls(fn)]
    golden["immersed_sphere"] = {"added_mass_heave": vals[0], "added_mass_surge": vals[4]}

    fn = funcs["test_floating_sphere_finite_freq"]
    calls = _isclose_calls(fn)
    golden["floating_sphere"] = {
        "omega_1": {"added_mass": ast.literal_eval(calls[0].args[1]),
                    "damping": ast.literal_eval(calls[1].args[1]),
                    "diffraction_force_polar": _complex_polar(calls[2].args[1])},
        "omega_2": {"added_mass": ast.literal_eval(calls[3].args[1]),
                    "damping": ast.literal_eval(calls[4].args[1]),
                    "diffraction_force_polar": _complex_polar(calls[5].args[1])},
    }
    fn = funcs["test_alien_sphere"]
    calls = _isclose_calls(fn)
    golden["alien_sphere"] = {"rho": 450.0, "g": 1.625, "omega": 1.0,
                              "added_mass": ast.literal_eval(calls[0].args[1]),
                              "damping": ast.literal_eval(calls[1].args[1]),
                              "diffraction_force_polar": _complex_polar(calls[2].args[1])}
    fn = funcs["test_floating_sphere_finite_depth"]
    calls = _isclose_calls(fn)
    # calls: A, B (omega 1), Kochin, F (omega 1), A, B (omega 2), F (omega 2)
    golden["floating_sphere_finite_depth"] = {
        "depth": 10.0,
        "omega_1": {"added_mass": ast.literal_eval(calls[0].args[1]),
                    "damping": ast.literal_eval(calls[1].args[1]),
                    "diffraction_force_polar": _complex_polar(calls[3].args[1])},
        "omega_2": {"added_mass": ast.literal_eval(calls[4].args[1]),
                    "damping": ast.literal_eval(calls[5].args[1]),
                    "diffraction_force_polar": _complex_polar(calls[6].args[1])},
    }
    fn = funcs["test_two_distant_spheres_in_finite_depth"]
    calls = _isclose_calls(fn)
    golden["two_spheres_finite_depth"] = {"depth": 10.0, "omega": 7.0, "radius": 0.5, "resolution": 4,
                                          "spacing": 20.0,
                                          "added_mass_surge": ast.literal_eval(calls[0].args[1]),
                                          "damping_surge": ast.literal_eval(calls[1].args[1])}
    fn = funcs["test_multibody"]
    for node in ast.walk(fn):
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name) \
                and node.targets[0].id == "data_from_nemoh_2":
            table = _literal(node.value)
    golden["multibody_sphere_cylinder"] = {
        "omega": 1.0,
        "dofs": ["cylinder_1__Surge", "cylinder_1__Heave", "sphere_0__Surge", "sphere_0__Heave"],
        "added_mass": [row[0::2] for row in table],
        "damping": [row[1::2] for row in table],
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
    with open(out, "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the capytaine source tree>")
    main(sys.argv[1])
