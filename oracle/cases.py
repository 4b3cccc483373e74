"""The case catalogue lives in tensorforge_b200.workloads (input builders only); this
module keeps the test-side import path `oracle.cases` working."""
from tensorforge_b200.workloads import *  # noqa: F401,F403
from tensorforge_b200.workloads import CASES, build, num_elements, ns_from_module  # noqa: F401
