"""The ground-sink test decks with particles placed to settle onto the
ground: every fluid cell of the first row above the ground gets a volume
fraction of 0.005 per class and a downward particle velocity of 0.5 m/s,
so that the sink (sink.f:46-121) acts from the first boundary call."""


def seeded_case(builder, edit=None, **kw):
    """The deck of `builder`, changed by edit(deck) when given, set up and
    seeded."""
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    deck = getattr(configs, builder)(**kw)
    if edit is not None:
        edit(deck)
    case = Case(deck)
    st, n = case.state, case.ncell
    plane = case.nx * (case.ny if case.is3d else 1)
    for c in range(n):
        if c // plane + 1 == 2 and case.flag[c] & 1:
            for q in range(case.nsolid):
                st["rlk"][q * n + c] += 0.005 * case.deck["density"][q]
                st["ws"][q * n + c] = -0.5
    return case
