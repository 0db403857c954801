function [g_w,a_max] = w_grad(u_w,geome_,finite_,gerjoii_,parame_)
% Drop-in for src/w/w_grad.m (reference adjoint semantics) via gj_mex.
g = gj_grid_(geome_,parame_,finite_);
[g_w,a_max] = gj_mex('w_grad', parame_.w.epsilon, parame_.w.sigma, g, ...
                     gerjoii_.w.s, gerjoii_.w.M, gerjoii_.w.wvlet_, ...
                     double(gerjoii_.w.e_2d), double(u_w));
g_w = single(g_w); a_max = single(a_max);
end
