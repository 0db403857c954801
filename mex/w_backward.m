function [g_e,g_s] = w_backward(geome_,parame_,finite_,gerjoii_)
% Backward half of the exact forward/backward pair via gj_mex: w_solve (the
% forward) gives gerjoii_.w.d_2d, w_fwd.m:34 the residual gerjoii_.w.e_2d, and
% this returns the exact adjoint of the forward map applied to that residual,
% dJ/d(epsilon_r) and dJ/d(sigma) of J = 0.5*||d - d_o||^2 for this shot (the
% role of w_grad.m after w_fwd in w_update_e.m:98 / w_update_s.m:77).
g = gj_grid_(geome_,parame_,finite_);
[g_e,g_s] = gj_mex('w_backward', parame_.w.epsilon, parame_.w.sigma, g, ...
                   double(gerjoii_.w.s), {gerjoii_.w.M}, gerjoii_.w.wvlet_, ...
                   {double(gerjoii_.w.e_2d)}, 1);
g_e = single(g_e); g_s = single(g_s);
end
