"""The C-ABI device context of the kernel-level GPU tests (artss_b200.Context)."""
from artss_b200 import Context  # noqa: F401
