function gerjoii_ = dc_gradient2_5d(parame_,finite_,gerjoii_)
% Drop-in for src/dc/dc_gradient2_5d.m via gj_mex: the library runs the forward
% and adjoint solves of all wavenumbers and returns the trimmed gradient.
[AB, I, MN, g] = gj_dc_src_(parame_,finite_,gerjoii_);
[gerjoii_.dc.g, d, e] = gj_mex('dc_gradient2_5d', parame_.dc.sigma_robin, g, AB, I, {MN}, ...
                               {finite_.dc.ky_w_}, [], {parame_.natu.dc.d});
gerjoii_.dc.d = d;
gerjoii_.dc.e_ = e;
end
