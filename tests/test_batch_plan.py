"""CPU checks of the batched-program planner (qlagpu_F3_batch_plan_program):
malformed programs are refused on the host, before any device work, with
QLAGPU_ERR_ARG and a message naming the field, the step and the fault.  The
stream bases are plain aligned addresses that nothing dereferences."""
import pytest

import qla_b200 as qla

X, M = 1 << 20, 1 << 21  # 16-B aligned addresses (never dereferenced: validation fails first)


@pytest.mark.parametrize("prog,words", [
    ({"n": 64, "streams": [dict(base=X, kind="D", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="lmult", a=0, b=0, store=1)]}, "a must be a colour matrix"),
    ({"n": 64, "streams": [dict(base=M, kind="M", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="lmult", a=0, b=qla.REG1, store=1)]}, "register read before"),
    ({"n": 64, "streams": [dict(base=X, kind="D", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="copy", a=0, store=1), dict(op="copy", a=0, store=1)]}, "more than one step"),
    ({"n": 64, "streams": [dict(base=X, index=X, kind="D", role="out")],
      "steps": [dict(op="copy", a=0, store=0)]}, "only IN streams"),
    ({"n": 64, "streams": [dict(base=X, kind="D", role="in"), dict(base=X, kind="H", role="out")],
      "steps": [dict(op="copy", a=0, store=1)]}, "another kind"),
    ({"n": 64, "streams": [dict(base=X, kind="D", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="copy", a=1, store=1)]}, "output of this launch"),
    ({"n": 64, "streams": [dict(base=X, kind="H", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="sprecon", eqop="peq", a=0, store=1)]}, "peq / meq needs"),
    ({"n": 64, "streams": [dict(base=X + 4, kind="D", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="copy", a=0, store=1)]}, "8-B aligned"),
    ({"n": 64, "streams": [dict(base=X, kind="D", role="in"), dict(base=X, kind="D", role="out")],
      "steps": [dict(op="copy", a=0)]}, "never stored"),
])
def test_malformed_programs_are_refused(prog, words):
    qla.clear_error()
    with pytest.raises(qla.QLAError) as e:
        qla.BatchProgramPlan([prog])
    assert words in str(e.value) and "field 0" in str(e.value), str(e.value)
    qla.clear_error()


def test_check_index_refuses_bad_arguments_without_a_gpu():
    qla.clear_error()
    assert qla.check_index(1 << 20, -1, 10)[0] == 4       # negative n
    assert qla.check_index(1 << 20, 10, -1)[0] == 4       # negative nsrc
    assert qla.check_index(0, 10, 10)[0] == 1             # NULL stream
    assert qla.check_index(0, 0, 10) == (0, -1)           # nothing to scan
    qla.clear_error()
