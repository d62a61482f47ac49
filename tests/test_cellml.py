"""CellML front end (cubie_b200.cellml.load_cellml_model).

The models are written here, in CellML 1.0 and 2.0, for these tests.  The
loaded systems are checked against the same equations given as strings
(symbolically, and by integrating both with the emulated kernel), plus the
loader's handling of connections, initial values given by name, piecewise
definitions, e-notation numbers, parameters and observables."""

import numpy as np
import pytest
import sympy as sp

FHN = ["dV = V - V**3 / 3 - w + I", "dw = (V + a - b * w) / tau"]

FHN_CELLML_10 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.0#" xmlns:cellml="http://www.cellml.org/cellml/1.0#"
       name="fhn_two_components">
  <units name="ms"><unit units="second" prefix="milli"/></units>
  <component name="environment">
    <variable name="time" units="ms" public_interface="out"/>
  </component>
  <component name="membrane">
    <variable name="time" units="ms" public_interface="in"/>
    <variable name="V" units="dimensionless" initial_value="-1.2" public_interface="out"/>
    <variable name="w_in" units="dimensionless" public_interface="in"/>
    <variable name="I" units="dimensionless" initial_value="0.5"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/>
        <apply><diff/><bvar><ci>time</ci></bvar><ci>V</ci></apply>
        <apply><plus/>
          <apply><minus/><ci>V</ci>
            <apply><divide/><apply><power/><ci>V</ci><cn cellml:units="dimensionless">3</cn></apply>
              <cn cellml:units="dimensionless">3</cn></apply></apply>
          <apply><minus/><ci>w_in</ci></apply>
          <ci>I</ci>
        </apply>
      </apply>
    </math>
  </component>
  <component name="recovery">
    <variable name="time" units="ms" public_interface="in"/>
    <variable name="V" units="dimensionless" public_interface="in"/>
    <variable name="w" units="dimensionless" initial_value="0.6" public_interface="out"/>
    <variable name="a" units="dimensionless" initial_value="0.7"/>
    <variable name="b" units="dimensionless" initial_value="0.8"/>
    <variable name="tau" units="ms" initial_value="1.25e1"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/>
        <apply><diff/><bvar><ci>time</ci></bvar><ci>w</ci></apply>
        <apply><divide/>
          <apply><minus/><apply><plus/><ci>V</ci><ci>a</ci></apply><apply><times/><ci>b</ci><ci>w</ci></apply></apply>
          <ci>tau</ci></apply>
      </apply>
    </math>
  </component>
  <connection><map_components component_1="environment" component_2="membrane"/>
    <map_variables variable_1="time" variable_2="time"/></connection>
  <connection><map_components component_1="environment" component_2="recovery"/>
    <map_variables variable_1="time" variable_2="time"/></connection>
  <connection><map_components component_1="membrane" component_2="recovery"/>
    <map_variables variable_1="V" variable_2="V"/>
    <map_variables variable_1="w_in" variable_2="w"/></connection>
</model>
"""

GATE_CELLML_20 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/2.0#" xmlns:cellml="http://www.cellml.org/cellml/2.0#" name="gate">
  <component name="main">
    <variable name="t" units="ms" interface="public"/>
    <variable name="x" units="dimensionless" initial_value="x0"/>
    <variable name="x0" units="dimensionless" initial_value="0.25"/>
    <variable name="V" units="mV" initial_value="-20"/>
    <variable name="k" units="per_ms" initial_value="3"/>
    <variable name="alpha" units="per_ms"/>
    <variable name="drive" units="dimensionless"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><ci>alpha</ci>
        <piecewise>
          <piece><apply><times/><cn cellml:units="per_ms" type="e-notation">2.5<sep/>-1</cn>
              <apply><exp/><apply><divide/><ci>V</ci><cn cellml:units="mV">10</cn></apply></apply></apply>
            <apply><lt/><ci>V</ci><cn cellml:units="mV">0</cn></apply></piece>
          <otherwise><apply><root/><degree><cn cellml:units="dimensionless">2</cn></degree><ci>k</ci></apply></otherwise>
        </piecewise>
      </apply>
      <apply><eq/><ci>drive</ci><apply><sin/><apply><times/><pi/><ci>t</ci></apply></apply></apply>
      <apply><eq/>
        <apply><diff/><bvar><ci>t</ci></bvar><ci>x</ci></apply>
        <apply><plus/>
          <apply><times/><ci>alpha</ci><apply><minus/><cn cellml:units="dimensionless">1</cn><ci>x</ci></apply></apply>
          <apply><times/><cn cellml:units="dimensionless">0.1</cn><ci>drive</ci></apply>
          <apply><minus/><apply><times/><ci>k</ci><ci>x</ci></apply></apply>
        </apply>
      </apply>
    </math>
  </component>
</model>
"""


def _write(tmp_path, text, name):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_fhn_components_and_connections(tmp_path):
    from cubie_b200 import create_ODE_system
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.cellml"), precision=np.float64,
                            parameters=["a", "tau"])
    assert ode.state_names == ["V", "w"]
    assert ode.initial_values == {"V": -1.2, "w": 0.6}
    assert ode.parameters == {"a": 0.7, "tau": 12.5}
    assert ode.constants == {"I": 0.5, "b": 0.8}
    ref = create_ODE_system(FHN, states={"V": -1.2, "w": 0.6}, parameters={"a": 0.7, "tau": 12.5},
                            constants={"I": 0.5, "b": 0.8}, precision=np.float64)
    names = {s.name: s for s in set().union(*[e.free_symbols for e in ref.derivatives.values()])}
    for st in ("V", "w"):
        mine = ode.derivatives[st].subs({s: names.get(s.name, s) for s in ode.derivatives[st].free_symbols})
        assert sp.simplify(mine - ref.derivatives[st]) == 0


def test_fhn_integrates_like_the_string_system(tmp_path):
    from host_emu.emu import run_emulated
    from cubie_b200 import Solver, create_ODE_system
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.cellml"), precision=np.float64,
                            parameters=["a", "b", "tau", "I"])
    ref = create_ODE_system(FHN, states={"V": -1.2, "w": 0.6}, parameters={"a": 0.7, "b": 0.8, "tau": 12.5, "I": 0.5},
                            precision=np.float64)
    rng = np.random.default_rng(3)
    x0 = np.stack([rng.uniform(-1, 1, 4), rng.uniform(-0.5, 0.5, 4)])
    p = np.stack([rng.uniform(0.5, 0.9, 4), rng.uniform(0.6, 1.0, 4), rng.uniform(8, 15, 4), rng.uniform(0.3, 0.6, 4)])
    out = []
    for sysm in (ode, ref):
        s = Solver(sysm, algorithm="dormand-prince-54", rtol=1e-9, atol=1e-9, save_every=1.0, output_types=["state"])
        out.append(run_emulated(s, x0, p, 20.0)["state"])
    np.testing.assert_allclose(out[0], out[1], rtol=1e-12, atol=1e-12)


def test_cellml2_piecewise_initial_by_name_and_observables(tmp_path):
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, GATE_CELLML_20, "gate.cellml"), precision=np.float64,
                            observables=["alpha"])
    assert ode.state_names == ["x"] and ode.initial_values == {"x": 0.25}
    assert ode.observable_names == ["alpha"]
    assert set(ode.constants) == {"x0", "V", "k"}
    d = ode.derivatives["x"]
    t = [s for s in d.free_symbols if s.name == "t"] or [sp.Symbol("t", real=True)]
    alpha = {s.name: e for s, e in ode.assignments}["alpha"]
    sub = {s: v for s in alpha.free_symbols | d.free_symbols for n, v in (("V", -20.0), ("k", 3.0)) if s.name == n}
    assert float(alpha.subs(sub)) == pytest.approx(0.25 * np.exp(-2.0))
    sub_pos = {s: (15.0 if s.name == "V" else 3.0) for s in alpha.free_symbols}
    assert float(alpha.subs(sub_pos)) == pytest.approx(np.sqrt(3.0))
    # dx/dt at x = 0.25, t = 0.5 with V = -20
    vals = {"x": 0.25, "t": 0.5, "V": -20.0, "k": 3.0}
    expr = d
    for s, e in ode.assignments:
        if s.name in ("alpha", "drive"):
            expr = expr.subs(s, e)
    got = float(expr.subs({s: vals[s.name] for s in expr.free_symbols}))
    want = 0.25 * np.exp(-2.0) * 0.75 + 0.1 * np.sin(np.pi * 0.5) - 3.0 * 0.25
    assert got == pytest.approx(want, rel=1e-12)


def test_loader_errors(tmp_path):
    from cubie_b200.cellml import load_cellml_model
    with pytest.raises(FileNotFoundError):
        load_cellml_model(tmp_path / "missing.cellml")
    with pytest.raises(ValueError, match=".cellml"):
        load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.xml"))
    with pytest.raises(ValueError, match="not constants"):
        load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.cellml"), parameters=["V"])
    with pytest.raises(ValueError, match="observable"):
        load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.cellml"), observables=["a"])


@pytest.mark.gpu
def test_cellml_model_solves_on_the_gpu_like_the_string_system(tmp_path, cuda_device):
    from cubie_b200 import Solver, create_ODE_system
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, FHN_CELLML_10, "fhn.cellml"), precision=np.float64,
                            parameters=["a", "b", "tau", "I"])
    ref = create_ODE_system(FHN, states={"V": -1.2, "w": 0.6}, parameters={"a": 0.7, "b": 0.8, "tau": 12.5, "I": 0.5},
                            precision=np.float64)
    rng = np.random.default_rng(4)
    x0 = np.stack([rng.uniform(-1, 1, 256), rng.uniform(-0.5, 0.5, 256)])
    p = np.stack([rng.uniform(0.5, 0.9, 256), rng.uniform(0.6, 1.0, 256), rng.uniform(8, 15, 256),
                  rng.uniform(0.3, 0.6, 256)])
    res = [Solver(sysm, algorithm="dormand-prince-54", rtol=1e-9, atol=1e-9, save_every=1.0,
                  output_types=["state"]).solve(x0, p, duration=20.0) for sysm in (ode, ref)]
    assert np.all(res[0].status_codes == 0)
    np.testing.assert_allclose(res[0].state, res[1].state, rtol=1e-10, atol=1e-12)


def test_cellml2_model_compiles_and_integrates(tmp_path):
    """The piecewise / sin / root model through code generation: NVRTC
    compiles it for sm_100a and the emulated kernel matches SciPy."""
    from scipy.integrate import solve_ivp as scipy_ivp
    from host_emu.emu import run_emulated
    from cubie_b200 import Solver, _native
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, GATE_CELLML_20, "gate.cellml"), precision=np.float64,
                            parameters=["V", "k"])
    s = Solver(ode, algorithm="dormand-prince-54", rtol=1e-10, atol=1e-10, save_every=0.5, output_types=["state"])
    gk = s._generate(s.kernel_spec(s._timing(2.0)))
    _native.compile_cubin(gk.source, _native.default_options(), use_cache=False)
    V = np.array([-20.0, 15.0])
    k = np.array([3.0, 1.5])
    got = run_emulated(s, np.full((1, 2), 0.25), np.stack([V, k]), 2.0)["state"][:, 0, :]

    def rhs(t, x, v, kk):
        alpha = 0.25 * np.exp(v / 10.0) if v < 0 else np.sqrt(kk)
        return [alpha * (1 - x[0]) + 0.1 * np.sin(np.pi * t) - kk * x[0]]

    for j in range(2):
        ref = scipy_ivp(rhs, (0, 2.0), [0.25], args=(V[j], k[j]), t_eval=np.arange(5) * 0.5, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got[:, j], ref.y[0], rtol=1e-8, atol=1e-9)


def test_cellml11_namespace_and_unsupported_elements(tmp_path):
    from cubie_b200.cellml import load_cellml_model
    v11 = FHN_CELLML_10.replace("cellml/1.0#", "cellml/1.1#")
    ode = load_cellml_model(_write(tmp_path, v11, "fhn11.cellml"))
    assert ode.state_names == ["V", "w"]
    imported = v11.replace('<component name="environment">',
                           '<import xmlns:xlink="http://www.w3.org/1999/xlink" xlink:href="other.cellml"/>'
                           '<component name="environment">')
    with pytest.raises(FileNotFoundError):               # imports resolve relative to the file
        load_cellml_model(_write(tmp_path, imported, "imp.cellml"))
    reset = GATE_CELLML_20.replace("</component>", "<reset variable=\"x\" test_variable=\"x\" order=\"1\"/></component>")
    with pytest.raises(NotImplementedError, match="reset"):
        load_cellml_model(_write(tmp_path, reset, "reset.cellml"))


UNITS_CELLML_11 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.1#" xmlns:cellml="http://www.cellml.org/cellml/1.1#" name="units">
  <units name="millisecond"><unit units="second" prefix="milli"/></units>
  <units name="millivolt"><unit units="volt" prefix="milli"/></units>
  <units name="per_volt"><unit units="volt" exponent="-1"/></units>
  <component name="env">
    <variable name="time" units="second" public_interface="out"/>
  </component>
  <component name="cell">
    <variable name="time" units="millisecond" public_interface="in"/>
    <variable name="V" units="millivolt" initial_value="-65" public_interface="out"/>
    <variable name="Vrest" units="millivolt" initial_value="-80"/>
    <variable name="tau" units="millisecond" initial_value="10"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><apply><diff/><bvar><ci>time</ci></bvar><ci>V</ci></apply>
        <apply><divide/><apply><minus/><ci>Vrest</ci><ci>V</ci></apply><ci>tau</ci></apply></apply>
    </math>
  </component>
  <component name="probe">
    <variable name="V" units="volt" public_interface="in"/>
    <variable name="Vv" units="volt"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><ci>Vv</ci><apply><times/><cn cellml:units="dimensionless">2</cn><ci>V</ci></apply></apply>
    </math>
  </component>
  <connection><map_components component_1="env" component_2="cell"/>
    <map_variables variable_1="time" variable_2="time"/></connection>
  <connection><map_components component_1="cell" component_2="probe"/>
    <map_variables variable_1="V" variable_2="V"/></connection>
</model>
"""


def test_cellml_units_convert_across_connections(tmp_path):
    """Time in seconds in one component and milliseconds in another, a
    voltage in millivolts read as volts elsewhere: the model variable keeps
    its defining occurrence's units and every other occurrence is scaled."""
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, UNITS_CELLML_11, "units.cellml"), precision=np.float64,
                            observables=["Vv"])
    V = sp.Symbol("V", real=True)
    assert ode.state_names == ["V"] and ode.initial_values["V"] == -65.0
    # dV/dt_ms = (Vrest - V) / tau_ms with t in seconds: 1000 x
    dv = ode.derivatives["V"].subs({sp.Symbol("Vrest", real=True): -80.0, sp.Symbol("tau", real=True): 10.0})
    assert sp.simplify(dv - 100 * (-80 - V)) == 0
    vv = dict((str(a), e) for a, e in ode.assignments)["Vv"]
    assert sp.simplify(vv - V / 500) == 0                  # 2 x (V mV in volts)
    bad = UNITS_CELLML_11.replace('<variable name="V" units="volt" public_interface="in"/>',
                                  '<variable name="V" units="second" public_interface="in"/>')
    with pytest.raises(ValueError, match="incompatible units"):
        load_cellml_model(_write(tmp_path, bad, "bad.cellml"), observables=["Vv"])


LIB_CELLML_11 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.1#" xmlns:cellml="http://www.cellml.org/cellml/1.1#" name="lib">
  <units name="per_second"><unit units="second" exponent="-1"/></units>
  <component name="decay">
    <variable name="t" units="second" public_interface="in" private_interface="out"/>
    <variable name="x" units="dimensionless" initial_value="2" public_interface="out"/>
    <variable name="k" units="per_second" private_interface="in"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><apply><diff/><bvar><ci>t</ci></bvar><ci>x</ci></apply>
        <apply><minus/><apply><times/><ci>k</ci><ci>x</ci></apply></apply></apply>
    </math>
  </component>
  <component name="rate">
    <variable name="k" units="per_second" initial_value="0.5" public_interface="out"/>
  </component>
  <group><relationship_ref relationship="encapsulation"/>
    <component_ref component="decay"><component_ref component="rate"/></component_ref></group>
  <connection><map_components component_1="decay" component_2="rate"/>
    <map_variables variable_1="k" variable_2="k"/></connection>
</model>
"""

MAIN_CELLML_11 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.1#" xmlns:cellml="http://www.cellml.org/cellml/1.1#"
       xmlns:xlink="http://www.w3.org/1999/xlink" name="main">
  <import xlink:href="lib.cellml">
    <component name="first_order" component_ref="decay"/>
    <units name="per_second" units_ref="per_second"/>
  </import>
  <component name="env">
    <variable name="time" units="second" public_interface="out"/>
    <variable name="y" units="dimensionless" initial_value="1"/>
    <variable name="x" units="dimensionless" public_interface="in"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><apply><diff/><bvar><ci>time</ci></bvar><ci>y</ci></apply><ci>x</ci></apply>
    </math>
  </component>
  <connection><map_components component_1="env" component_2="first_order"/>
    <map_variables variable_1="time" variable_2="t"/>
    <map_variables variable_1="x" variable_2="x"/></connection>
</model>
"""


def test_cellml_import_brings_the_encapsulated_components(tmp_path):
    """A component imported from another document (CellML 1.1), with the
    component it encapsulates and the connection between them."""
    from cubie_b200.cellml import load_cellml_model
    _write(tmp_path, LIB_CELLML_11, "lib.cellml")
    ode = load_cellml_model(_write(tmp_path, MAIN_CELLML_11, "main.cellml"), precision=np.float64,
                            parameters=["k"])
    assert sorted(ode.state_names) == ["x", "y"] and ode.parameters == {"k": 0.5}
    x, y, k = (sp.Symbol(n, real=True) for n in ("x", "y", "k"))
    assert sp.simplify(ode.derivatives["x"] + k * x) == 0 and sp.simplify(ode.derivatives["y"] - x) == 0
    cyc = LIB_CELLML_11.replace('name="lib">', 'name="lib" xmlns:xlink="http://www.w3.org/1999/xlink">'
                                '<import xlink:href="main.cellml"/>')
    _write(tmp_path, cyc, "lib.cellml")
    with pytest.raises(ValueError, match="cycle"):
        load_cellml_model(tmp_path / "main.cellml")


TEMP_CELLML_11 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.1#" xmlns:cellml="http://www.cellml.org/cellml/1.1#" name="temp">
  <units name="per_second"><unit units="second" exponent="-1"/></units>
  <units name="fahrenheit"><unit units="kelvin" multiplier="0.5555555555555556" offset="255.37222222222223"/></units>
  <component name="env">
    <variable name="time" units="second" public_interface="out"/>
  </component>
  <component name="body">
    <variable name="time" units="second" public_interface="in"/>
    <variable name="T" units="kelvin" initial_value="310" public_interface="out"/>
    <variable name="Ta" units="celsius" public_interface="in"/>
    <variable name="k" units="per_second" initial_value="0.1"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><apply><diff/><bvar><ci>time</ci></bvar><ci>T</ci></apply>
        <apply><times/><ci>k</ci><apply><minus/><apply><plus/><ci>Ta</ci>
          <cn cellml:units="kelvin">273.15</cn></apply><ci>T</ci></apply></apply></apply>
    </math>
  </component>
  <component name="room">
    <variable name="Ta" units="celsius" initial_value="20" public_interface="out"/>
  </component>
  <component name="probe">
    <variable name="T" units="celsius" public_interface="in"/>
    <variable name="Tc" units="celsius"/>
    <variable name="Tf" units="fahrenheit" public_interface="out"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><ci>Tc</ci><ci>T</ci></apply>
      <apply><eq/><ci>Tf</ci><ci>T</ci></apply>
    </math>
  </component>
  <component name="reader">
    <variable name="Tf" units="kelvin" public_interface="in"/>
    <variable name="Tk" units="kelvin"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><ci>Tk</ci><ci>Tf</ci></apply>
    </math>
  </component>
  <connection><map_components component_1="env" component_2="body"/>
    <map_variables variable_1="time" variable_2="time"/></connection>
  <connection><map_components component_1="room" component_2="body"/>
    <map_variables variable_1="Ta" variable_2="Ta"/></connection>
  <connection><map_components component_1="body" component_2="probe"/>
    <map_variables variable_1="T" variable_2="T"/></connection>
  <connection><map_components component_1="probe" component_2="reader"/>
    <map_variables variable_1="Tf" variable_2="Tf"/></connection>
</model>
"""


def test_cellml_offset_units_convert_affinely(tmp_path):
    """A temperature held in kelvin and read in celsius elsewhere shifts by
    273.15; a CellML 1.1 unit with an offset (Fahrenheit over kelvin)
    converts through its multiplier and offset when read across a
    connection; the ODE in kelvin is unchanged by the offsets of the other
    occurrences."""
    from cubie_b200.cellml import load_cellml_model
    ode = load_cellml_model(_write(tmp_path, TEMP_CELLML_11, "temp.cellml"), precision=np.float64,
                            observables=["Tc", "Tf", "Tk"])
    T = sp.Symbol("T", real=True)
    assert ode.state_names == ["T"] and ode.initial_values["T"] == 310.0
    asg = dict((str(a), e) for a, e in ode.assignments)
    # dT/dt = k ((Ta_C + 273.15) - T) with the room at 20 C
    dT = ode.derivatives["T"].subs({sp.Symbol("k", real=True): 0.1, sp.Symbol("Ta", real=True): 20.0})
    assert abs(float(dT.subs(T, 300.0)) - 0.1 * (293.15 - 300.0)) < 1e-12
    # probe: T (kelvin) read in celsius
    assert abs(float(asg["Tc"].subs(T, 310.0)) - 36.85) < 1e-12
    # within a component an equation relates values in their own units
    # (no conversion): Tf holds the probe's celsius number as fahrenheit
    assert abs(float(asg["Tf"].subs(T, 310.0)) - 36.85) < 1e-12
    # the reader sees Tf in kelvin: 36.85 F = 36.85 * 5/9 + 255.372 K
    tk = asg["Tk"].subs(sp.Symbol("Tf", real=True), asg["Tf"]).subs(T, 310.0)
    assert abs(float(tk) - (36.85 * 0.5555555555555556 + 255.37222222222223)) < 1e-9
    # an offset on a compound unit is rejected
    bad = TEMP_CELLML_11.replace('<units name="fahrenheit"><unit units="kelvin" multiplier="0.5555555555555556" '
                                 'offset="255.37222222222223"/></units>',
                                 '<units name="fahrenheit"><unit units="kelvin" exponent="2" offset="1"/></units>')
    with pytest.raises(ValueError, match="offset"):
        load_cellml_model(_write(tmp_path, bad, "bad_temp.cellml"), observables=["Tc", "Tf", "Tk"])


GHK_CELLML_10 = """<?xml version="1.0"?>
<model xmlns="http://www.cellml.org/cellml/1.0#" xmlns:cellml="http://www.cellml.org/cellml/1.0#" name="ghk">
  <units name="ms"><unit units="second" prefix="milli"/></units>
  <units name="mV"><unit units="volt" prefix="milli"/></units>
  <units name="per_ms"><unit units="second" prefix="milli" exponent="-1"/></units>
  <units name="mV_per_ms"><unit units="mV"/><unit units="ms" exponent="-1"/></units>
  <component name="environment">
    <variable name="time" units="ms" public_interface="out"/>
  </component>
  <component name="membrane">
    <variable name="time" units="ms" public_interface="in"/>
    <variable name="V" units="mV" initial_value="-65" public_interface="out"/>
    <variable name="m" units="dimensionless" initial_value="0.05"/>
    <variable name="alpha_m" units="per_ms"/>
    <math xmlns="http://www.w3.org/1998/Math/MathML">
      <apply><eq/><ci>alpha_m</ci>
        <apply><divide/>
          <apply><times/><cn cellml:units="per_ms">0.1</cn>
            <apply><plus/><ci>V</ci><cn cellml:units="mV">40</cn></apply></apply>
          <apply><minus/><cn cellml:units="dimensionless">1</cn>
            <apply><exp/><apply><divide/>
              <apply><minus/><apply><plus/><ci>V</ci><cn cellml:units="mV">40</cn></apply></apply>
              <cn cellml:units="mV">10</cn></apply></apply></apply></apply></apply>
      <apply><eq/><apply><diff/><bvar><ci>time</ci></bvar><ci>m</ci></apply>
        <apply><times/><ci>alpha_m</ci><apply><minus/><cn cellml:units="dimensionless">1</cn><ci>m</ci></apply></apply></apply>
      <apply><eq/><apply><diff/><bvar><ci>time</ci></bvar><ci>V</ci></apply>
        <apply><minus/><ci>m</ci></apply></apply>
    </math>
  </component>
  <connection><map_components component_1="environment" component_2="membrane"/>
    <map_variables variable_1="time" variable_2="time"/></connection>
</model>
"""


def test_cellml_removable_ghk_singularity_is_rewritten(tmp_path):
    """alpha_m = 0.1 (V + 40) / (1 - exp(-(V + 40) / 10)) is 0 / 0 at
    V = -40 as written; with the membrane voltage detected, the rewritten
    rate is finite there (its limit, 1) and equal to the original away from
    it; with fix_singularities=False the expression is kept as written."""
    from cubie_b200.cellml import load_cellml_model
    path = _write(tmp_path, GHK_CELLML_10, "ghk.cellml")
    V = sp.Symbol("V", real=True)
    fixed = load_cellml_model(path, precision=np.float64, observables=["alpha_m"])
    raw = load_cellml_model(path, precision=np.float64, observables=["alpha_m"], fix_singularities=False)
    a_fixed = dict((str(a), e) for a, e in fixed.assignments)["alpha_m"]
    a_raw = dict((str(a), e) for a, e in raw.assignments)["alpha_m"]
    f_fixed = sp.lambdify(V, a_fixed, "math")
    f_raw = sp.lambdify(V, a_raw, "math")
    assert abs(f_fixed(-40.0) - 1.0) < 1e-15
    with pytest.raises(ZeroDivisionError):
        f_raw(-40.0)
    # against the written rate evaluated in 50-digit arithmetic (in FP64
    # the written form itself loses about eps / |U| near the singularity;
    # closer than about 1e-4 the rounding of its decimal constants, which
    # moves the numerator's zero by ~1e-15, decides the written value)
    for v in (-40.0 - 3e-4, -40.0 + 2e-3, -40.5, -65.0, 10.0):
        exact = float(a_raw.subs(V, sp.Float(repr(v), 50)).evalf(50))
        assert abs(f_fixed(v) - exact) <= 1e-10 * abs(exact), v
    assert abs(f_fixed(-40.0 + 1e-9) - (1.0 + 5e-11)) < 1e-14      # the limit's first-order term
    # an explicitly named voltage that does not exist is an error
    with pytest.raises(ValueError, match="membrane voltage"):
        load_cellml_model(path, voltage_variable="U")
