"""Numpy model of the pruned five-pass operator schedule (test infrastructure).

Mirrors the index arithmetic of vie_fft_b200/csrc/vie_operator.cuh -- radix
plans, in-place DIF/DIT stages with digit-reversed spectra, the exact split
of every zero-padded length-2N axis into two length-N transforms, the
natural-order z spectra, the per-axis P/Q symbol tables and the folded Green
octant -- so that the formulation itself can be checked against the oracle
on the CPU, independently of the CUDA code.
"""
import numpy as np

PI = 3.1415926535897932384626433832795
Z0 = 120 * PI


def plan(n):
    rad=[]; m=n
    while m%16==0: rad.append(16); m//=16
    if m%8==0: rad.append(8); m//=8
    elif m%4==0: rad.append(4); m//=4
    elif m%2==0: rad.append(2); m//=2
    p=3
    while m>1:
        if p*p>m: rad.append(m); m=1; break
        while m%p==0: rad.append(p); m//=p
        p+=2
    return rad

def perm_of(n,rad):
    perm=np.zeros(n,int)
    for m in range(n):
        rem=m; pos=0; span=n
        for R in rad:
            q=rem%R; rem//=R; span//=R; pos+=q*span
        perm[m]=pos
    return perm

def dif(x, rad, inv=False):
    # in-place DIF (fwd) on last axis, digit reversed output; inverse DIT
    x=x.copy(); n=x.shape[-1]
    tw=np.exp(-2j*np.pi*np.arange(2*n)/(2*n))
    if not inv:
        L=n
        for R in rad:
            m=L//R
            for b in range(n//L):
                for j in range(m):
                    idx=[b*L+j+r*m for r in range(R)]
                    v=x[...,idx]
                    W=np.exp(-2j*np.pi*np.outer(np.arange(R),np.arange(R))/R)
                    y=v@W  # y[q]=sum_r v[r] W[r,q]
                    for q in range(R):
                        if j: y[...,q]*=tw[(2*j*q*(n//L))%(2*n)]
                    x[...,idx]=y
            L=m
    else:
        m=1
        for R in reversed(rad):
            L=m*R
            for b in range(n//L):
                for j in range(m):
                    idx=[b*L+j+q*m for q in range(R)]
                    v=x[...,idx].copy()
                    for q in range(R):
                        if j: v[...,q]*=np.conj(tw[(2*j*q*(n//L))%(2*n)])
                    W=np.exp(2j*np.pi*np.outer(np.arange(R),np.arange(R))/R)
                    x[...,idx]=v@W
            m=L
    return x

def fwd_split(x, n, rad):  # x [...,n] -> [...,2n] slots (h*n+p)
    tw=np.exp(-2j*np.pi*np.arange(n)/(2*n))
    e=dif(x,rad); o=dif(x*tw,rad)
    return np.concatenate([e,o],-1)
def inv_split(X, n, rad):
    tw=np.exp(-2j*np.pi*np.arange(n)/(2*n))
    e=dif(X[...,:n],rad,True); o=dif(X[...,n:],rad,True)
    return e+np.conj(tw)*o

def slot_k(n, rad, natural):
    if natural: return np.arange(2*n)
    perm=perm_of(n,rad); dr=np.zeros(n,int); dr[perm]=np.arange(n)
    s=np.arange(2*n); h=(s>=n).astype(int); p=s-h*n
    return 2*dr[p]+h

def emulate(g, green_full, eps, flags, x, conj):
    nx,ny,nz=g.shape; d=[g.dx,g.dy,g.dz]; k0=g.k0; M=8*nx*ny*nz
    rads=[plan(nx),plan(ny),plan(nz)]
    J=x.copy()
    # validity
    J[0,nx-1,:,:]=0; J[1,:,ny-1,:]=0; J[2,:,:,nz-1]=0
    # F1 natural order z
    Xz=fwd_split(J,nz,rads[2])  # [3,nx,ny,2nz] slot order h*n+p
    kz_slot=slot_k(nz,rads[2],False)
    Xnat=np.zeros_like(Xz); Xnat[...,kz_slot]=Xz   # natural
    # F2 along y
    Xy=fwd_split(np.moveaxis(Xnat,2,-1),ny,rads[1])  # [3,nx,2nz,2ny]
    # F3 along x
    Xx=fwd_split(np.moveaxis(Xy,1,-1),nx,rads[0])    # [3,2nz,2ny,2nx]
    kx=slot_k(nx,rads[0],False); ky=slot_k(ny,rads[1],False); kz=np.arange(2*nz)
    # octant green from full spectrum
    oct_=green_full[:nx+1,:ny+1,:nz+1]
    fold=lambda k,n: np.where(k<=n,k,2*n-k)
    G=oct_[fold(kx,nx)[None,None,:], fold(ky,ny)[None,:,None], fold(kz,nz)[:,None,None]]  # [2nz,2ny,2nx]
    Gs=1j*Z0/(k0*M)*G
    def tabs(k,n,delta):
        th=2*PI*k/(2*n); c=np.cos(th); s=np.sin(th)
        dp=(1-c)+1j*s; dm=(c-1)+1j*s
        if not conj: return dp/delta, dm
        return np.conj(dm), np.conj(dp)/delta
    Px,Qx=tabs(kx,nx,d[0]); Py,Qy=tabs(ky,ny,d[1]); Pz,Qz=tabs(kz,nz,d[2])
    P=[Px[None,None,:],Py[None,:,None],Pz[:,None,None]]; Q=[Qx[None,None,:],Qy[None,:,None],Qz[:,None,None]]
    if conj: Gs=np.conj(Gs)
    rho=sum(P[s]*Xx[s] for s in range(3))
    E=np.stack([Gs*(k0*k0*d[f]*Xx[f]+Q[f]*rho) for f in range(3)])
    # inverse x
    Ex=inv_split(E,nx,rads[0])          # [3,2nz,2ny,nx]
    Ey=inv_split(np.moveaxis(Ex,-1,1),ny,rads[1])  # [3,nx,2nz,ny]
    Ezn=np.moveaxis(Ey,-1,2)            # [3,nx,ny,2nz] natural kz
    Ezs=Ezn[...,kz_slot]                # to slot order
    Y=inv_split(Ezs,nz,rads[2])         # [3,nx,ny,nz]
    # diag
    w=1/(eps-1)
    out=np.zeros_like(Y)
    for f in range(3):
        ws=np.zeros(g.shape,complex)
        sl=[slice(None)]*3; sl[f]=slice(0,g.shape[f]-1); sl=tuple(sl)
        sh=[slice(None)]*3; sh[f]=slice(1,None); sh=tuple(sh)
        ws[sl]=w[sh]+w[sl]
        dc=-d[f]*Z0/(2*k0)
        coef=1j*dc*ws
        if conj: coef=np.conj(coef)
        out[f]=(Y[f]+coef*J[f])*flags[f]
    return out

