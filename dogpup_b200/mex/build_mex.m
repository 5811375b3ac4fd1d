% Builds dogpup_b200's MATLAB gateways with mexcuda (interleaved complex).
% Run from this folder after building libdogpup_b200.so one level up
% (python -m dogpup_b200.build).  The first three replace the reference's
% cuda_lib mex files of the same names; put this folder on the MATLAB path
% ahead of cuda_lib.  bicgstab_fsai_mex is the one-call solve for fluGPU.
here = fileparts(mfilename('fullpath'));
pkg = fileparts(here);
inc = ['-I' fullfile(fileparts(pkg), 'include')];
lib = {['-L' pkg], '-ldogpup_b200', ['LDFLAGS=$LDFLAGS -Wl,-rpath,' pkg]};
gw = {'smv_mexgateway.cpp', 'smv_mex'; ...
      'FSAImv_mexgateway.cpp', 'FSAImv_mex'; ...
      'FSAIP_mexgateway.cpp', 'FSAIP_gen_mex'; ...
      'bicgstab_fsai_mexgateway.cpp', 'bicgstab_fsai_mex'};
for i = 1:size(gw, 1)
    mexcuda('-R2018a', inc, fullfile(here, gw{i, 1}), lib{:}, '-output', fullfile(here, gw{i, 2}));
end
