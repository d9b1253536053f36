function UaRestartToV7(RestartFile, OutFile)
%UaRestartToV7  Restart file of a forward run -> the MAT v7 layout uasource_b200 reads.
%
%   UaRestartToV7(RestartFile, OutFile)
%
% WriteForwardRunRestartFile.m:25 saves MUA, BCs, F, l, ... as MAT v7.3 (HDF5), where F, BCs
% and l are classdef objects (UaFields, BoundaryConditions, UaLagrangeVariables) that only MATLAB
% can decode.  This writes the same variables with those objects as plain structs, in MAT v7,
% for uasource_b200.restart.load_restart (MUA.coordinates, MUA.connectivity; the nodal F fields;
% the fixed-node BC lists, 1-based as in Ua; l.ubvb; CtrlVarInRestartFile.time and .dt).

S = load(RestartFile, 'CtrlVarInRestartFile', 'MUA', 'BCs', 'F', 'l');

MUA = struct('coordinates', S.MUA.coordinates, 'connectivity', S.MUA.connectivity);

F = struct();
fnames = {'h', 'S', 'B', 'rho', 'AGlen', 'n', 'C', 'm', 'ub', 'vb', 'as', 'ab', 'rhow', 'g', 'alpha'};
for k = 1:numel(fnames)
    if isprop(S.F, fnames{k}) && ~isempty(S.F.(fnames{k}))
        F.(fnames{k}) = double(S.F.(fnames{k}));
    end
end

BCs = struct();
bnames = {'ubFixedNode', 'ubFixedValue', 'vbFixedNode', 'vbFixedValue', 'hFixedNode', 'hFixedValue'};
for k = 1:numel(bnames)
    if isprop(S.BCs, bnames{k}) && ~isempty(S.BCs.(bnames{k}))
        BCs.(bnames{k}) = double(S.BCs.(bnames{k}));
    end
end

l = struct('ubvb', []);
if isprop(S.l, 'ubvb')
    l.ubvb = double(S.l.ubvb);
end

CtrlVarInRestartFile = struct('time', 0, 'dt', 0);
if isfield(S.CtrlVarInRestartFile, 'time'), CtrlVarInRestartFile.time = S.CtrlVarInRestartFile.time; end
if isfield(S.CtrlVarInRestartFile, 'dt'), CtrlVarInRestartFile.dt = S.CtrlVarInRestartFile.dt; end

save(OutFile, 'MUA', 'BCs', 'F', 'l', 'CtrlVarInRestartFile', '-v7');
end
