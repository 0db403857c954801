function gerjoii_ = w_solve(geome_,parame_,finite_,gerjoii_)
% Drop-in for src/w/w_solve.m: same signature, same outputs, computed by the
% B200 library through gj_mex.  The model is taken unpadded (parame_.w.epsilon,
% parame_.w.sigma); the library pads it as w_exp2pml.m does.
g = gj_grid_(geome_,parame_,finite_);
[d,u,Jz] = gj_mex('w_solve', parame_.w.epsilon, parame_.w.sigma, g, ...
                  gerjoii_.w.s, gerjoii_.w.M, gerjoii_.w.wvlet_);
gerjoii_.w.d_2d = single(d);
gerjoii_.w.u_2d = single(u);
gerjoii_.w.Jy = single(Jz);
end
