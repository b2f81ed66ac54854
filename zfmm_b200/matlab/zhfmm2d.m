function [pot,grad] = zhfmm2d(eps,zk,ns,zsrc,ifcharge,charge,ifdipole,dipstr,dipvec,nt,ztarg,ifpgh,isep)
% ZHFMM2D on the GPU through libzfmm_b200 (argument order of the
% reference's zhfmm2d.mw @function line).  Calls the gateway zhfmm2dmex built
% from zfmm_b200_mex.c by build_mex.sh, with the argument and size lists of
% the mwrap calling convention; library errors are raised as MATLAB errors.
pot = complex(zeros(nt,1));
grad = complex(zeros(2,nt));
ifprint = 0;
mex_id_ = 'zhfmm2d(i double[x], i dcomplex[x], i int[x], i dcomplex[xx], i int[x], i dcomplex[x], i int[x], i dcomplex[x], i dcomplex[xx], io dcomplex[x], io dcomplex[xx], i int[x], i dcomplex[xx], i int[x], i int[x], i int[x])';
[pot, grad] = zhfmm2dmex(mex_id_, eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, nt, ztarg, ifpgh, isep, ifprint, 1, 1, 1, 2, ns, 1, ns, 1, ns, 2, ns, nt, 2, nt, 1, 2, nt, 1, 1, 1);
end
