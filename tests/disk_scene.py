"""Seeded synthetic post-impact scenes (SI) for the disk measurement tests: the package's generator with the test
constants (a remnant ball, a ring of orbiting debris, escaping particles and clumps placed to exercise each gate of
the Moon-candidate test: bound outside the Roche limit, bound inside it, hot and unbound)."""
from botheadstudios_b200.ic import SCENE_CLUMPS as CLUMPS, SCENE_R as R, post_impact_scene as scene  # noqa: F401
from botheadstudios_b200.materials import G_SI as G, eos_table  # noqa: F401


def eos():
    return eos_table()
