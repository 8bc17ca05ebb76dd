"""cfd_plugin C ABI semantics that need no GPU (the reference's
zerork_cfd_plugin.cpp / optionable.cpp behaviour): defaults, option
round-trips, options-file keys, status codes for null handles/pointers."""
import ctypes as C

import pytest

from zerork_b200.plugin import Plugin, PluginError, plugin_lib


def test_defaults_match_reference_manager():
    p = Plugin()
    # zerork_reactor_manager.cpp:49-101
    assert p.get_double("rel_tol") == 1.0e-8
    assert p.get_double("abs_tol") == 1.0e-20
    assert p.get_int("max_steps") == 5000
    assert p.get_double("max_dt") == 0.05
    assert p.get_double("nonlinear_convergence_coeff") == 0.05
    assert p.get_double("step_limiter") == 1.0e22
    assert p.get_int("cvode_num_retries") == 5
    assert p.get_double("cvode_retry_absolute_tolerance_adjustment") == 0.1
    assert p.get_double("min_mass_fraction") == 1.0e-30
    assert p.get_int("sort_reactors") == 1
    assert p.get_string("mech_filename") == "mech.dat"
    # reactor model: constant volume, temperature always solved
    assert p.get_int("constant_volume") == 1
    assert p.get_int("always_solve_temperature") == 1
    assert p.get_double("solve_temperature_threshold") == 2.0
    assert p.get_double("delta_temperature_ignition") == 0.0


def test_option_roundtrip_and_unknown():
    p = Plugin()
    p.set_option("max_steps", 123)
    p.set_option("rel_tol", 1e-6)
    p.set_option("any_new_name", 7)  # setters accept any name
    assert p.get_int("max_steps") == 123 and p.get_double("rel_tol") == 1e-6
    assert p.get_int("any_new_name") == 7
    with pytest.raises(PluginError) as e:
        p.get_int("not_an_option")
    assert e.value.code == 8  # OPTION_NOT_DEFINED


def test_options_file(tmp_path):
    f = tmp_path / "opts.yml"
    f.write_text("relative_tolerance: 1.0e-06\nabsolute_tolerance: 1.0e-18\nmax_steps: 3000\n"
                 "reactor_timing_log: reactor.log   # comment\n\nnonlinear_convergence_coeff: 0.1\n")
    p = Plugin()
    p.read_options_file(f)
    assert p.get_double("rel_tol") == 1e-6 and p.get_double("abs_tol") == 1e-18
    assert p.get_int("max_steps") == 3000
    assert p.get_string("reactor_timing_log_filename") == "reactor.log"
    assert p.get_double("nonlinear_convergence_coeff") == 0.1
    f2 = tmp_path / "reactor.yml"
    f2.write_text("constant_volume: 0\nalways_solve_temperature: 0\n"
                  "solve_temperature_threshold: 5.0\n")
    p.read_options_file(f2)
    assert p.get_int("constant_volume") == 0 and p.get_int("always_solve_temperature") == 0
    assert p.get_double("solve_temperature_threshold") == 5.0
    bad = tmp_path / "bad.yml"
    bad.write_text("max_steps: lots\n")
    with pytest.raises(PluginError) as e:
        p.read_options_file(bad)
    assert e.value.code == 6  # FAILED_OPTIONS_PARSE
    with pytest.raises(PluginError) as e:
        p.read_options_file(tmp_path / "missing.yml")
    assert e.value.code == 6


def test_null_handle_and_pointer_statuses():
    L = plugin_lib()
    assert L.zerork_reactor_load_mechanism(None) == 1
    assert L.zerork_reactor_solve(0, 0.0, 1e-3, 1, None, None, None, None) == 1
    assert L.zerork_reactor_free(None) == 1
    p = Plugin()
    assert L.zerork_reactor_set_mechanism_files(None, None, p.h) == 2  # INVALID_FILENAME
    assert L.zerork_reactor_read_options_file(None, p.h) == 2
    assert L.zerork_reactor_set_aux_field_pointer(1, None, p.h) == 4  # INVALID_POINTER
    x = (C.c_double * 4)()
    assert L.zerork_reactor_set_aux_field_pointer(42, C.addressof(x), p.h) == 3  # INVALID_FIELD_NAME
    assert L.zerork_reactor_set_reactor_ids(None, p.h) == 4


def test_solve_zero_reactors_is_noop_after_load(c1):
    """n_reactors = 0 returns success once a mechanism is loadable; on a
    machine without a GPU, loading reports an error instead of falling back."""
    from conftest import have_gpu
    p = Plugin(*c1[1])
    L = plugin_lib()
    rc = L.zerork_reactor_load_mechanism(p.h)
    if have_gpu():
        assert rc == 0
    else:
        assert rc == 99


def test_bad_mechanism_status(tmp_path, c1):
    from conftest import have_gpu
    if not have_gpu():
        pytest.skip("mechanism upload needs a GPU")
    m = tmp_path / "bad.mech"
    m.write_text("ELEMENTS\nH\nEND\nSPECIES\nH2\nEND\nREACTIONS\nH2 <=> HX 1 0 0\nEND\n")
    p = Plugin(m, c1[1][1])
    with pytest.raises(PluginError) as e:
        p.load_mechanism()
    assert e.value.code == 5  # FAILED_MECHANISM_PARSE
