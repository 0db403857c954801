function [gerjoii_,finite_] = dc_fwd2_5d(parame_,finite_,gerjoii_)
% Drop-in for src/dc/dc_fwd2_5d.m via gj_mex: data d, residual e_ and the
% stacked potential u of the current source (all wavenumbers in one call, the
% Robin coefficients computed by the library).  The per-wavenumber fields u_k
% are not returned; dc_gradient2_5d.m in this folder does not need them.
[AB, I, MN, g] = gj_dc_src_(parame_,finite_,gerjoii_);
[d, u] = gj_mex('dc_fwd2_5d', parame_.dc.sigma_robin, g, AB, I, {MN}, {finite_.dc.ky_w_}, []);
gerjoii_.dc.d = d;
gerjoii_.dc.e_ = d - parame_.natu.dc.d;
gerjoii_.dc.u = reshape(u, [finite_.dc.nx, finite_.dc.nz]);
end
