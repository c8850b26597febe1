"""The jax.ffi route (chromatix_b200.jaxffi): runs only where jax and its FFI
headers are installed.  The custom call returns what the torch path returns
for the same field, and jax.grad through its custom_vjp matches the torch
autograd gradient (the same adjoint kernels)."""

import numpy as np
import pytest

from tests.helpers import rand_field

pytestmark = pytest.mark.gpu


def _need_jax():
    from chromatix_b200 import jaxffi

    if not jaxffi.available():
        pytest.skip("jax (with its FFI headers) is not installed")
    return jaxffi


@pytest.mark.parametrize("mode", ["full", "same"])
def test_ffi_call_matches_torch_path_and_gradient(mode):
    jaxffi = _need_jax()
    import jax
    import jax.numpy as jnp
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    u = rand_field((64, 48), seed=3)
    out_j = np.asarray(jaxffi.asm_propagate(jnp.asarray(u), 25.0, 1.33, 16, 0.3, 0.532, mode=mode))
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    out_t = cf.asm_propagate(cx.Field.build(ut, 0.3, 0.532), 25.0, 1.33, 16, mode=mode).u
    np.testing.assert_array_equal(out_j, out_t.detach().cpu().numpy())
    w = (np.random.default_rng(4).standard_normal(out_j.shape) + 1j).astype(np.complex64)
    g_j = jax.grad(lambda v: jnp.real(jnp.vdot(jnp.asarray(w), jaxffi.asm_propagate(v, 25.0, 1.33, 16, 0.3, 0.532,
                                                                                     mode=mode))))(jnp.asarray(u))
    torch.real(torch.sum(torch.conj(torch.as_tensor(w, device="cuda")) * out_t)).backward()
    # jax returns the conjugate of torch's gradient convention for complex inputs
    np.testing.assert_allclose(np.conj(np.asarray(g_j)), ut.grad.cpu().numpy(), rtol=1e-5, atol=1e-5)
