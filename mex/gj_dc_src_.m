function [AB, I, MN, g] = gj_dc_src_(parame_,finite_,gerjoii_)
% One DC source in the gateway's arguments, from the reference's structs:
% AB (1 x 2, 1-based) the +I and -I nodes of the source vector gerjoii_.dc.s
% (dc_electrodes.m:54-55), I its current, MN (nd x 2) the +1 and -1 columns of
% each row of the measuring operator gerjoii_.dc.M (dc_M.m), g the grid struct
% (robin, and the spacings of finite_.dc.DELTAS, do_grid.m).
s = gerjoii_.dc.s;
a = find(s > 0, 1);
b = find(s < 0, 1);
AB = [a b];
I = full(s(a));
[r, c, v] = find(gerjoii_.dc.M);
MN = zeros(size(gerjoii_.dc.M, 1), 2);
MN(r(v > 0), 1) = c(v > 0);
MN(r(v < 0), 2) = c(v < 0);
g = struct('robin', parame_.dc.robin, 'dx', finite_.dc.DELTAS(1,1,1), 'dz', finite_.dc.DELTAS(1,1,2));
end
