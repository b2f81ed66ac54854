function [pot,grad] = zl3devaldirect(nt,ztarg,ns,zsrc,charge,dipstr,dipvec,ifcharge,ifdipole,ifpgh)
% ZL3DEVALDIRECT on the GPU through libzfmm_b200 (argument order of the
% reference's zl3devaldirect.mw @function line).  Calls the gateway zl3devaldirectmex built
% from zfmm_b200_mex.c by build_mex.sh, with the argument and size lists of
% the mwrap calling convention; library errors are raised as MATLAB errors.
pot = complex(zeros(nt,1));
grad = complex(zeros(3,nt));
mex_id_ = 'zl3devaldirect(i int[x], i dcomplex[xx], i int[x], i dcomplex[xx], i dcomplex[x], i dcomplex[x], i dcomplex[xx], i int[x], io dcomplex[x], io dcomplex[xx], i int[x], i int[x])';
[pot, grad] = zl3devaldirectmex(mex_id_, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad, ifdipole, ifpgh, 1, 3, nt, 1, 3, ns, ns, ns, 3, ns, 1, nt, 3, nt, 1, 1);
end
