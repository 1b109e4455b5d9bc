"""Where the reference's source tree lies: the one setting every build
recipe and test that reads it uses.  Override with the environment variable
MVR_REFERENCE_ROOT; the tree is optional (absent on machines that only run
the prebuilt oracle libraries)."""
import os

REF_ROOT = os.environ.get("MVR_REFERENCE_ROOT", "/root/reference")


def ref_path(*parts: str) -> str:
    return os.path.join(REF_ROOT, *parts)
