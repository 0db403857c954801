function [gerjoii_,finite_] = dc_fwd2_5d(parame_,finite_,gerjoii_)
% Drop-in for src/dc/dc_fwd2_5d.m via gj_mex: data d, residual e_, the
% stacked potential u and the per-wavenumber potentials u_k of the current
% source (all wavenumbers in one call, the Robin coefficients computed by the
% library), the fields dc_fwd2_5d.m:56-61 sets.
[AB, I, MN, g] = gj_dc_src_(parame_,finite_,gerjoii_);
[d, u, u_k] = gj_mex('dc_fwd2_5d', parame_.dc.sigma_robin, g, AB, I, {MN}, {finite_.dc.ky_w_}, []);
gerjoii_.dc.d = d;
gerjoii_.dc.e_ = d - parame_.natu.dc.d;
gerjoii_.dc.u = reshape(u, [finite_.dc.nx, finite_.dc.nz]);
gerjoii_.dc.u_k = u_k;
end
