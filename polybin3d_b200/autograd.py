"""Differentiable estimator numerators: the Q-maps of the Monte Carlo Fisher matrices are
vector-Jacobian products of these functions.

For the power spectrum (PolyBin3D/pspec.py:613-686, trivial S^-1, data = m * d)

    num_{l b}(d) = 1/2 V/N^6 sum_k deg Theta_b L_{2l} |rfftn(m d) / W|^2
    d num_{l b} / d d = V/N^3 * m * irfftn(Theta_b L_{2l} rfftn(m d) / W^2)

so the reference's Q_{l b} = rfftn(m irfftn(Theta_b L_{2l} rfftn(m a)))  (pspec.py:443-456)
is (N^3/V) rfftn(d num_{l b}/d d) at d = a.  The backward is one pass of the binned-weight
filter kernel (pb_binned_filter) with the cotangent as per-bin weights, one c2r and one mask
product.  For the local sightline multipole l is the cross spectrum of x = rfftn(m d)/W with
H_l[x] = sum_m Y_lm(k) FT[Y_lm(r) IFT x]; its gradient adds the adjoint transform, the same
two parts as the reference's local Q-maps (pspec.py:456-486).

For the bispectrum (PolyBin3D/bspec.py:895-983, no linear term) the numerator is
V/(N^3 sym_i) sum_x g_b1 g_b2 g_{l,b3} with g_{l,b} = irfftn(Theta_b L_l rfftn(m d) / W);
its derivative is the sum over the three legs of irfftn(Theta_leg L_leg / W FT[product of the
other two maps]) times m, the same construction as the reference's Q-maps (bspec.py:600-640).
The backward recomputes the bin-filtered maps (nothing is stored by the forward), sums, in
real space, the products of the other two maps of every leg that ends on the same (bin,
multipole) with pb_bilinear_maps (one map per leg instead of one per pair of maps),
transforms those, and gathers them into one spectrum with the accumulating spectral filter.  Maps, products and their transforms live
on the dealiased map grid, which is exact for every frequency inside the bins.  With the
local sightline the l > 0 maps are IFT(Theta_b H_l x): their legs are gathered through the bin
filter alone, one spectrum per l, and the adjoint H_l^dag applied once per l.
"""
import numpy as np
import torch

from . import _native as nat


def _mask_of(est, dtype=torch.float64):
    if est.const_mask:
        return None
    if dtype == torch.float64:
        return est._mask_device()
    return est.base.to_device_grid(('mask', id(est)), lambda: est.mask, dtype)


def _settle():
    """Backward runs on autograd's device thread.  On B200 a cuFFT transform issued from that
    thread while the forward's kernels were still running returned CUFFT_EXEC_FAILED (seen at
    512^3, where the forward's contraction runs for tens of ms); waiting for the stream first
    avoids it.  The wait costs nothing measurable next to a backward pass."""
    torch.cuda.current_stream().synchronize()


# device bytes the Bk backward may hold in pair products and their spectra at once
KEY_CHUNK_BYTES = 16 << 30


class PkNumerator(torch.autograd.Function):
    """num = PkNumerator.apply(d, pspec): the unwindowed numerator of data m*d as a
    differentiable FP64 device tensor (N_bins,); global and local sightlines (odd l too)."""

    @staticmethod
    def _spectrum(ps, d):
        """x = rfftn(m d) / W."""
        b = ps.base
        m = _mask_of(ps)
        y = d if m is None else nat.elementwise(nat.PB_EW_MUL, d, m)
        xk = b.fft_r2c(y)
        b.n_FFTs_forward += 1
        if b.pixel_window != 'none':
            w = b.to_device_grid('window', lambda: b.pixel_window_grid, torch.float64)
            nat.spectral_filter(b.grid, nat.PB_F64, xk, xk, [(0, -1.0, np.inf, 0, 0, 1.0, -1)], w=w)
        return xk

    @staticmethod
    def forward(ctx, d, ps):
        b = ps.base
        d = d.to(torch.float64).contiguous()
        ctx.ps = ps
        ctx.save_for_backward(d)
        xk = PkNumerator._spectrum(ps, d)
        out = torch.empty(ps.N_bins, dtype=torch.float64, device=b.device)
        scale = 0.5 * b.volume / float(b.gridsize.prod()) ** 2
        if b.sightline == 'global' or ps.Nl == 1:
            nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_ABS2, xk, None, 1, ps.k_bins, ps._ells(ps.Nl), scale, out,
                           b.ws)
            return out
        # local sightline (pspec.py:643-680): multipole l crosses x with p_l H_l[x],
        # H_l[x] = sum_m Y_lm(k) FT[Y_lm(r) IFT x], p_l = -i for odd l, 1 for even l
        Nk = ps.Nk
        nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_ABS2, xk, None, 1, ps.k_bins, [(0, 0)], scale, out[:Nk], b.ws)
        x_real = b.to_real(xk)
        for li in range(1, ps.Nl):
            l = li * (2 - ps.odd_l)
            lm = b.harmonics.apply_fourier(x_real, l)
            if l % 2:
                lm = lm * (-1j)
            nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_CROSS, xk, lm, 1, ps.k_bins, [(0, 0)], scale,
                           out[li * Nk:(li + 1) * Nk], b.ws)
        return out

    @staticmethod
    def _local_backward(ps, d, coef):
        """Gradient of sum_{l b} g_{l b} num_{l b} for the local sightline.  With
        num_{l b} = 1/2 V/N^6 sum_k Theta_b Re(x conj(p_l H_l x)) and x = F(m d)/W, the
        gradient of Re<x, Theta p H x> in x is Theta p H x + conj(p) H^dag Theta x, where
        H^dag v = FT[sum_m Y_lm(r) IFT(Y_lm(k) v)] (the second part of the reference's local
        Q-maps, pspec.py:466-483), and d/dd = m F^dag W^-1: grad = V/N^6 m c2r(S / W),
        S = Theta_g0 x + sum_l 1/2 (p Theta_gl H_l x + conj(p) H_l^dag Theta_gl x),
        Theta_g the bin filter weighted by the cotangent."""
        b = ps.base
        harm = b.harmonics
        xk = PkNumerator._spectrum(ps, d)
        S = torch.empty_like(xk)
        nat.binned_filter(b.grid, xk, S, ps.k_bins, [0], coef[0:1])
        x_real = b.to_real(xk)
        R = torch.zeros_like(d)
        t = torch.empty_like(xk)
        u = torch.empty_like(xk)
        for li in range(1, ps.Nl):
            l = li * (2 - ps.odd_l)
            nat.binned_filter(b.grid, harm.apply_fourier(x_real, l), t, ps.k_bins, [0], coef[li:li + 1], scale=0.5)
            S.add_(t * (-1j) if l % 2 else t)
            # H^dag Theta_g x; conj(p) = i goes in before the inverse transform, where it makes
            # the odd-l spectrum Hermitian again
            nat.binned_filter(b.grid, xk, u, ps.k_bins, [0], coef[li:li + 1], scale=0.5 / b.nreal)
            if l % 2:
                u.mul_(1j)
            yr = harm._grid('r', l, torch.float64)
            yk = harm._grid('k', l, torch.float64)
            for mi in range(yr.shape[0]):
                v = u * yk[mi]
                b.n_FFTs_reverse += 1
                R.addcmul_(b.fft_c2r(v), yr[mi])
        b.n_FFTs_forward += 1
        S.add_(b.fft_r2c(R))
        if b.pixel_window != 'none':
            w = b.to_device_grid('window', lambda: b.pixel_window_grid, torch.float64)
            nat.spectral_filter(b.grid, nat.PB_F64, S, S, [(0, -1.0, np.inf, 0, 0, 1.0, -1)], w=w)
        S.mul_(b.volume / float(b.gridsize.prod()) ** 2)
        b.n_FFTs_reverse += 1
        grad = b.fft_c2r(S)
        m = _mask_of(ps)
        if m is not None:
            grad = nat.elementwise(nat.PB_EW_MUL, grad, m, out=grad)
        return grad

    @staticmethod
    def backward(ctx, g):
        _settle()
        ps = ctx.ps
        b = ps.base
        (d,) = ctx.saved_tensors
        coef = g.to(torch.float64).reshape(ps.Nl, ps.Nk).contiguous()
        if b.sightline == 'local' and ps.Nl > 1:
            return PkNumerator._local_backward(ps, d, coef), None
        m = _mask_of(ps)
        y = d if m is None else nat.elementwise(nat.PB_EW_MUL, d, m)
        xk = b.fft_r2c(y)
        b.n_FFTs_forward += 1
        w = None
        if b.pixel_window != 'none':
            w = b.to_device_grid('window', lambda: b.pixel_window_grid, torch.float64)
        spec = torch.empty_like(xk)
        nat.binned_filter(b.grid, xk, spec, ps.k_bins, [2 * li for li in range(ps.Nl)], coef, w=w,
                          wpow=-2 if w is not None else 0, scale=b.volume / float(b.gridsize.prod()) ** 2)
        grad = b.fft_c2r(spec)
        b.n_FFTs_reverse += 1
        if m is not None:
            grad = nat.elementwise(nat.PB_EW_MUL, grad, m, out=grad)
        return grad, None


class BkNumerator(torch.autograd.Function):
    """num = BkNumerator.apply(d, bspec): the unwindowed numerator (no linear term) of data
    m*d as a differentiable FP64 device tensor (N_bins,); global and local sightlines.  Maps, transforms and the gradient
    run in the base's precision (FP64, or FP32 with precision='mixed'); the cubic sums are
    FP64 either way."""

    @staticmethod
    def _maps(bs, d):
        b = bs.base
        m = _mask_of(bs, d.dtype)
        y = d if m is None else nat.elementwise(nat.PB_EW_MUL, d, m)
        xk = b.fft_r2c(y)
        b.n_FFTs_forward += 1
        w = None
        if b.pixel_window != 'none':
            w = b.to_device_grid(('bk_invwin', id(bs)), lambda: bs._inv_window(), d.dtype)
        return bs._g_maps(xk, w, 1.0)

    @staticmethod
    def forward(ctx, d, bs):
        if not hasattr(bs, 'sym_factor'):
            bs._compute_symmetry_factor()
        ctx.in_dtype = d.dtype
        d = d.to(bs.base.real_dtype).contiguous()
        ctx.bs = bs
        ctx.save_for_backward(d)
        G = BkNumerator._maps(bs, d)
        B3 = bs._contract('b3', G, G, G, bs._triplet_index())
        norm = torch.as_tensor(bs.base.volume / float(bs.base.gridsize.prod()) / bs.sym_factor, device=d.device)
        return B3 * norm

    @staticmethod
    def backward(ctx, g):
        _settle()
        bs = ctx.bs
        b = bs.base
        (d,) = ctx.saved_tensors
        rd = d.dtype
        prec = nat.precision_of(rd)
        cd = torch.complex128 if rd == torch.float64 else torch.complex64
        G = BkNumerator._maps(bs, d)  # recomputed, not stored
        Mdims = tuple(int(n) for n in G.shape[1:])
        nks = bs.Nk_squeeze
        ks = bs.k_bins_squeeze
        ab = bs.all_bins
        gam = g.to(torch.float64).cpu().numpy()
        N3 = float(b.gridsize.prod())
        M3 = float(np.prod(Mdims))
        # coefficient of triplet i: V / (sym_i N^3) * (N^3/M^3) [map-grid transform] / N^3 [c2r]
        coef = gam * b.volume / (bs.sym_factor * N3 * M3)
        legs = {}
        keys = {}

        def key_of(i, j):
            return keys.setdefault((i, j), len(keys))

        for t, (b1, b2, b3, l) in enumerate(ab.tolist()):
            if coef[t] == 0.0:
                continue
            c3 = (l // 2) * nks + b3
            for (kk, C, lc) in ((key_of(b2, c3), b1, 0), (key_of(b1, c3), b2, 0), (key_of(b1, b2), b3, l)):
                legs[(kk, C, lc)] = legs.get((kk, C, lc), 0.0) + coef[t]
        # local sightline: the l > 0 maps are IFT(Theta_b H_l x), so a leg ending on (C, l > 0)
        # goes through the bin filter alone into an accumulator per l, and H_l^dag is applied
        # once per l below (H_l^dag v = FT[sum_m Y_lm(r) IFT(Y_lm(k) v)])
        local = b.sightline == 'local' and bs.lmax > 0
        n_acc = 1 + (bs.lmax // 2 if local else 0)
        grad_spec = torch.zeros((n_acc,) + b.nhalf_shape, dtype=cd, device=b.device)
        if keys:
            # one real-space map per leg (bin C, multipole lc): the coefficient-weighted sum of
            # the products of the other two maps of every triplet ending on it (pb_bilinear_maps);
            # then one forward transform per leg and one accumulating filter into the gradient
            pairs = sorted(keys, key=keys.get)
            outs = sorted({(C, lc) for (kk, C, lc) in legs})
            opos = {oc: n for n, oc in enumerate(outs)}
            tl = [(opos[(C, lc)], pairs[kk][0], pairs[kk][1], v) for (kk, C, lc), v in legs.items()]
            plan = nat.BilinearPlan(G.shape[0], len(outs), [t[0] for t in tl], [t[1] for t in tl],
                                    [t[2] for t in tl], [t[3] for t in tl], b.device)
            R = plan.maps(G)
            del G
            per_out = R[0].numel() * R.element_size() * 2
            chunk = int(max(1, min(len(outs), KEY_CHUNK_BYTES // per_out)))
            for o0 in range(0, len(outs), chunk):
                o1 = min(len(outs), o0 + chunk)
                FT = b.fft_r2c(R[o0:o1])
                b.n_FFTs_forward += o1 - o0
                entries = [(n - o0, ks[C], ks[C + 1], 0 if local else lc, 0, 1.0, 0)
                           for n, (C, lc) in enumerate(outs[o0:o1], o0)]
                dst = [lc // 2 if local else 0 for (C, lc) in outs[o0:o1]]
                nat.spectral_filter(b.grid_of(Mdims), prec, FT, grad_spec, entries, accumulate=True,
                                    src_stride=FT[0].numel(), out_n=[int(n) for n in b.gridsize], dst=dst)
                del FT
        if n_acc > 1:
            harm = b.harmonics
            R = torch.zeros((1,) + tuple(int(n) for n in b.gridsize), dtype=rd, device=b.device)
            for li in range(1, n_acc):
                yr = harm._grid('r', 2 * li, rd)
                yk = harm._grid('k', 2 * li, rd)
                for mi in range(yr.shape[0]):
                    b.n_FFTs_reverse += 1
                    R[0].addcmul_(b.fft_c2r((grad_spec[li] * yk[mi]).contiguous()), yr[mi])
            b.n_FFTs_forward += 1
            grad_spec = grad_spec[0:1] + b.fft_r2c(R) * (1.0 / N3)
        if b.pixel_window != 'none':
            w = b.to_device_grid('window', lambda: b.pixel_window_grid, rd)
            nat.spectral_filter(b.grid, prec, grad_spec, grad_spec, [(0, -1.0, np.inf, 0, 0, 1.0, -1)], w=w)
        grad = b.fft_c2r(grad_spec)[0]
        b.n_FFTs_reverse += 1
        m = _mask_of(bs, rd)
        if m is not None:
            grad = nat.elementwise(nat.PB_EW_MUL, grad, m, out=grad)
        return grad.to(ctx.in_dtype), None


def pk_numerator(ps, d):
    """Differentiable unwindowed power-spectrum numerator of data m*d (FP64 device tensor)."""
    return PkNumerator.apply(d, ps)


def bk_numerator(bs, d):
    """Differentiable unwindowed bispectrum numerator (no linear term) of data m*d."""
    return BkNumerator.apply(d, bs)


def q_maps_pk(ps, d):
    """All N_bins Q-maps (N^3/V) rfftn(d num_i/d d) at d, as rows of a complex128 tensor;
    equal to the reference's Q_{l b} of pspec.py:443-456 when d is the GRF in real space."""
    b = ps.base
    d = d.to(torch.float64).contiguous().requires_grad_(True)
    out = torch.empty((ps.N_bins,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
    num = pk_numerator(ps, d)
    for i in range(ps.N_bins):
        (gi,) = torch.autograd.grad(num[i], d, retain_graph=i + 1 < ps.N_bins)
        out[i] = b.fft_r2c(gi.contiguous()) * (float(b.gridsize.prod()) / b.volume)
    return out
