"""CPU: the C-ABI library loads, exports every entry point include/*.h declares,
its structure layouts match the Python bindings, and the host-only parts of the
ABI (configuration front-end, validation, error reporting) behave like the
reference's (no device work is launched here)."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\*?\s*(qk_[a-z_0-9]+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol(qk):
    lib = C.CDLL(str(ROOT / "quantkos_b200" / "libquantkos_b200.so"))
    names = _declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same surface
    from quantkos_b200._lib import SIGNATURES
    assert sorted(SIGNATURES) == names


def test_struct_layouts_match_c(tmp_path, qk):
    from quantkos_b200 import _lib as L
    src = tmp_path / "sz.c"
    src.write_text(textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "quantkos_b200.h"
        int main(void) {
          printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(qk_contract), sizeof(qk_config),
                 sizeof(qk_result), sizeof(qk_greeks), sizeof(qk_timing), sizeof(qk_serve_stats), sizeof(qk_payoff),
                 offsetof(qk_contract, payoffs), offsetof(qk_config, paths_file), offsetof(qk_result, p),
                 sizeof(qk_tune_report), offsetof(qk_tune_report, best_ms), sizeof(qk_serve_options),
                 offsetof(qk_serve_options, reserve_mib), sizeof(qk_serve_record), offsetof(qk_serve_record, est_ms));
          return 0;
        }"""))
    exe = tmp_path / "sz"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(L.Contract), C.sizeof(L.Config), C.sizeof(L.Result), C.sizeof(L.Greeks), C.sizeof(L.Timing),
            C.sizeof(L.ServeStats), C.sizeof(L.Payoff), L.Contract.payoffs.offset, L.Config.paths_file.offset,
            L.Result.p.offset, C.sizeof(L.TuneReport), L.TuneReport.best_ms.offset, C.sizeof(L.ServeOptions),
            L.ServeOptions.reserve_mib.offset, C.sizeof(L.ServeRecord), L.ServeRecord.est_ms.offset]
    assert got == want


def test_cxx_header_compiles(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "quantkos_b200.hpp"\nint main() { quantkos::Config::UInputs u; (void)u; return 0; }\n')
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{ROOT / 'include'}", str(src)], check=True)


def test_version_and_no_device_error(qk):
    lib = qk.lib.lib()
    assert lib.qk_version().startswith(b"quantkos_b200")
    import torch
    if not torch.cuda.is_available():
        h = C.c_void_p()
        assert lib.qk_create(0, C.byref(h)) == qk.lib.QK_ERR_NO_DEVICE
        assert b"no CUDA device" in lib.qk_last_error()


CONFIG_YAML = """
# Example input in the reference's format
Market:
  Price: 8.0      # spot
  Variance: 0.0625
  r: 0.1
  q: 0.0

Options:
  OptionType:  Asian   # comment after value
  OptionRight:  Call
  StrikePrice: 10.

Model:
  Heston:
    k: 5.0
    theta: 0.16
    sigma: 0.9
    rho: 0.1

Numerics:
  Scheme: ImplicitMilstein

Time:
  T_End: 0.25
  Inp_DT: 0.00025

MC:
  Normalize_prices : true
  N_Paths: 1000000
  Batch_Size: 0
  RNG_Seed: 88471920573105
  Max_VRAM_MB: 256
  Max_CPU_RAM_MB: 8000
  compute_delta_et_gamma: true
  compute_vega_et_vomma: true
  compute_vanna: true
  compute_rho: true
  compute_theta: true
  compute_vega : false        # unknown key: ignored, as by the reference
  analyze_risk_neutral_payoff_distribution: false

Output:
  out_dir: ""
  Name_Paths_Out_File: ""
  Name_Log_File: ""
  Format: BIN
"""


def test_parser_reads_reference_format(qk):
    u = qk.Parser.parse_string(CONFIG_YAML)
    assert u.S0 == 8.0 and u.v0 == 0.0625 and u.r == 0.1 and u.K == 10.0
    assert u.opt_type == qk.ASIAN and u.opt_right == qk.CALL
    assert u.model == qk.HESTON and u.heston_k == 5.0 and u.heston_sigma == 0.9 and u.heston_rho == 0.1
    assert u.scheme == qk.IMPLICIT_MILSTEIN
    assert u.n_steps == 1000 and abs(u.dt - 0.00025) < 1e-15  # TimeConfig::validate
    assert u.n_paths == 1_000_000 and u.seed == 88471920573105 and u.normalize == 1
    assert u.greeks_mask == qk.GREEK_ALL
    assert u.paths_file == "" and u.out_dir == ""
    k, g = u.to_contract()
    assert k.n_steps == 1000 and k.payoffs[0].type == qk.ASIAN and g.mask == 31 and g.bump_vol == 0.01


def test_parser_time_grid_rounding(qk):
    y = CONFIG_YAML.replace("Inp_DT: 0.00025", "Inp_DT: 0.0027397260273972603").replace("T_End: 0.25", "T_End: 1.")
    u = qk.Parser.parse_string(y)
    assert u.n_steps == 365


@pytest.mark.parametrize("mutate,needle", [
    (lambda y: y.replace("Market:", "Markets:"), "Mandatory block 'Market' missing"),
    (lambda y: y.replace("OptionType:  Asian", "OptionType:  Bermudan"), "Invalid value 'Bermudan'"),
    (lambda y: y.replace("  Heston:\n", "  Heston:\n    k: 1.0\n  Bates:\n    k: 1.0\n"), "both Heston and Bates"),
    (lambda y: y.replace("  Heston:", "  SABR:"), "non implemented model"),
    (lambda y: y.replace("Price: 8.0", "Price: -8.0"), "must be positive"),
    (lambda y: y.replace("RNG_Seed: 88471920573105", "RNG_Seed: 0"), "seed cannot be 0"),
    (lambda y: y.replace("Inp_DT: 0.00025", "Inp_DT: 0.5"), "must be smaller that total time"),
    (lambda y: y.replace("rho: 0.1", "rho: 1.5"), "rho must fall within"),
    (lambda y: y.replace("StrikePrice: 10.", "StrikePrice: 0.0001"), "too close to zero"),
    (lambda y: y.replace("Format: BIN", "Format: TXT"), "Unsupported output format"),
    (lambda y: y.replace("Normalize_prices : true", "Normalize_prices : maybe"), "must be a boolean"),
])
def test_parser_errors_match_reference(qk, mutate, needle):
    with pytest.raises(ValueError) as ei:
        qk.Parser.parse_string(mutate(CONFIG_YAML))
    assert needle in str(ei.value)


def test_parse_file_missing(qk, tmp_path):
    with pytest.raises(ValueError, match="File not found"):
        qk.Parser.parse(str(tmp_path / "nope.yaml"))


def test_validate_greek_bumps(qk):
    k = qk.make_contract(v0=0.04)
    g = qk.make_greeks(bump_vol=0.5)  # larger than sqrt(v0)
    lib = qk.lib.lib()
    assert lib.qk_validate(C.byref(k), C.byref(g)) == qk.lib.QK_ERR_INVALID_ARG
    assert b"volatility_absolute_bump_size" in lib.qk_last_error()
    g = qk.make_greeks()
    assert lib.qk_validate(C.byref(k), C.byref(g)) == qk.lib.QK_OK
    k.n_paths = 0
    assert lib.qk_validate(C.byref(k), None) == qk.lib.QK_ERR_INVALID_ARG


def test_parser_engine_extension_keys(qk):
    """Extension keys (absent from the reference's configs; defaults keep its behaviour)."""
    u = qk.Parser.parse_string(CONFIG_YAML)
    assert u.precision == qk.FP64 and u.engine == 0 and u.antithetic == 0 and u.stream == 0
    y = CONFIG_YAML.replace("  RNG_Seed: 88471920573105",
                            "  RNG_Seed: 88471920573105\n  Precision: FP32\n  Engine: batch\n  Antithetic: true\n"
                            "  Stream: 7\n  Vega_Mode: 1")
    u = qk.Parser.parse_string(y)
    assert u.precision == qk.FP32 and u.engine == 1 and u.antithetic == 1 and u.stream == 7 and u.vega_mode == 1
    k, g = u.to_contract()
    assert k.antithetic == 1 and k.precision == qk.FP32 and k.stream == 7 and g.vega_mode == 1
