C     SENGA_GPU: ISO_C_BINDING interface of libsenga_gpu.so for the
C     reference's Fortran driver (src/senga2.f). A host that keeps its
C     COMMON blocks builds this module with its own sources and calls the
C     device path in place of the routines it replaces (the call sites are
C     listed in INTEGRATION.md and in senga_gpu_drv.f beside this file).
C
C     Every BIND(C) type mirrors one struct of include/senga_gpu.h member by
C     member; C arrays [a][b][c] appear here as (c,b,a). The table bounds
C     equal the header's SENGA_* constants, which equal the reference's
C     PARAMETERs (src/com_senga2.h:80-98,181-187), NSPCMX and NSTPMX those
C     of its largest shipped case (src/casefiles/68step/com_senga2.h:74): a
C     host compiled with smaller tables fills the leading part of each. A CPU test of the
C     repository (tests/test_fortran_binding.py) parses this file and the
C     header and checks member order, types and extents against each other.
C     Every entry point returns 0 on success and a positive senga_status
C     code otherwise; SENGA_LAST_ERROR gives the message.
      MODULE SENGA_GPU
      USE ISO_C_BINDING
      IMPLICIT NONE
      INTEGER, PARAMETER :: SNSPCM = 18, SNSTPM = 68, SNTINM = 2
      INTEGER, PARAMETER :: SNCOFM = 7, SNSSMX = 10, SNBDYM = 10
      INTEGER, PARAMETER :: SNLLMX = 10, SNDCFM = 4, SNCFRM = 6
      INTEGER, PARAMETER :: SNOBC = 0, SNBOUN = 1, SNPERI = 2
C     ITNDEX arrays: (NSPEC + 14)/15 words per point, words slowest
      INTEGER, PARAMETER :: SNSPIM = 15
C     COMMON/CHEMIC after CHEMIN (src/com_senga2.h:121-178)
      TYPE, BIND(C) :: SENGA_CHEM
        INTEGER(C_INT) :: NSPEC, NSTEP, NBODY, NGIBB, NLIND, NTROE
        INTEGER(C_INT) :: NSRIF
        INTEGER(C_INT) :: NTINT(SNSPCM)
        INTEGER(C_INT) :: NCOFCP(SNTINM, SNSPCM)
        INTEGER(C_INT) :: NCPOLY(SNTINM, SNSPCM)
        INTEGER(C_INT) :: NCPOM1(SNTINM, SNSPCM)
        INTEGER(C_INT) :: NCENTH(SNTINM, SNSPCM)
        INTEGER(C_INT) :: NCENPY(SNTINM, SNSPCM)
        INTEGER(C_INT) :: NSSLEN(SNSTPM), NRSLEN(SNSTPM)
        INTEGER(C_INT) :: NPSLEN(SNSTPM)
        INTEGER(C_INT) :: NRCLEN(SNSTPM), NPCLEN(SNSTPM)
        INTEGER(C_INT) :: NSSPEC(SNSSMX, SNSTPM)
        INTEGER(C_INT) :: NRSPEC(SNSSMX, SNSTPM)
        INTEGER(C_INT) :: NPSPEC(SNSSMX, SNSTPM)
        INTEGER(C_INT) :: NRCPEC(SNSSMX, SNSTPM)
        INTEGER(C_INT) :: NPCPEC(SNSSMX, SNSTPM)
        INTEGER(C_INT) :: MBLIST(SNSTPM), MGLIST(SNSTPM)
        INTEGER(C_INT) :: MLLIST(SNSTPM)
        INTEGER(C_INT) :: MTLIST(SNSTPM), MSLIST(SNSTPM)
        REAL(C_DOUBLE) :: PREFGB, ALAMDA
        REAL(C_DOUBLE) :: TINTLO(SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: TINTHI(SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMOLCP(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMOLGB(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMASCP(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMASCT(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMASCH(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: AMASCS(SNCOFM, SNTINM, SNSPCM)
        REAL(C_DOUBLE) :: RPARAM(3, SNSTPM)
        REAL(C_DOUBLE) :: RCLIND(4, SNLLMX)
        REAL(C_DOUBLE) :: RCTROE(12, SNLLMX)
        REAL(C_DOUBLE) :: RCSRIF(8, SNLLMX)
        REAL(C_DOUBLE) :: DIFFMU(SNSSMX, SNSTPM)
        REAL(C_DOUBLE) :: DIFFMW(SNSSMX, SNSTPM)
        REAL(C_DOUBLE) :: CRSPEC(SNSSMX, SNSTPM)
        REAL(C_DOUBLE) :: CPSPEC(SNSSMX, SNSTPM)
        REAL(C_DOUBLE) :: EFFY3B(SNSPCM, SNBDYM)
        REAL(C_DOUBLE) :: WMOLAR(SNSPCM), OVWMOL(SNSPCM)
        REAL(C_DOUBLE) :: RGSPEC(SNSPCM)
        REAL(C_DOUBLE) :: CLEWIS(SNSPCM), OLEWIS(SNSPCM)
      END TYPE
C     COMMON/DIFFUS after DIFFIN (src/com_senga2.h:189-214)
      TYPE, BIND(C) :: SENGA_DIFF
        INTEGER(C_INT) :: FLMAVT, NCODIF, NCOTDR, NCOVIS, NCOCON
        REAL(C_DOUBLE) :: PDIFGB, TDIFGB
        REAL(C_DOUBLE) :: DIFFCO(SNDCFM, SNSPCM, SNSPCM)
        REAL(C_DOUBLE) :: TDRCCO(SNDCFM, SNSPCM, SNSPCM)
        REAL(C_DOUBLE) :: WILKO1(SNSPCM, SNSPCM)
        REAL(C_DOUBLE) :: WILKO2(SNSPCM, SNSPCM)
        REAL(C_DOUBLE) :: VISCCO(SNDCFM, SNSPCM)
        REAL(C_DOUBLE) :: CONDCO(SNDCFM, SNSPCM)
      END TYPE
C     cont.dat's grid, domain, end conditions and time step of one box
      TYPE, BIND(C) :: SENGA_CONFIG
        INTEGER(C_INT) :: NX, NY, NZ
        REAL(C_DOUBLE) :: XGDLEN, YGDLEN, ZGDLEN
        INTEGER(C_INT) :: NEND(6)
        REAL(C_DOUBLE) :: TSTEP
        INTEGER(C_INT) :: ADAPTIVE, DEVICE
      END TYPE
C     RADCIN's radiation tables (src/radcin.f:80-220)
      TYPE, BIND(C) :: SENGA_RADN
        INTEGER(C_INT) :: NSPRAD
        INTEGER(C_INT) :: NSPRID(SNSPCM)
        INTEGER(C_INT) :: NKPRAD(SNSPCM)
        REAL(C_DOUBLE) :: AKPRAD(SNCFRM, SNSPCM)
        REAL(C_DOUBLE) :: TREFRN
      END TYPE
C     NSCBC x faces: kinds 11 (I1 inflow), 12 (I2 inflow), 13 (I3
C     inflow), 14 (I4 inflow, x-left), 21 (O1 outflow), 31 (W1
C     adiabatic no-slip wall), 32 (W2 isothermal no-slip wall) and
C     parameters (T_IN: TRIN of an I2 inflow, the I4 target; T_WALL:
C     RXLPRM(1), RXRPRM(1) of W2 walls; NRIETA: RXLPRC(1..6) of I4)
      TYPE, BIND(C) :: SENGA_NSCBC
        INTEGER(C_INT) :: XL, XR
        REAL(C_DOUBLE) :: U_IN, RHO_IN
        REAL(C_DOUBLE) :: Y_IN(SNSPCM)
        REAL(C_DOUBLE) :: P_INF, SIGMA, ETA
        INTEGER(C_INT) :: PIO, BET_LOCAL
        REAL(C_DOUBLE) :: T_IN
        REAL(C_DOUBLE) :: T_WALL(2)
        REAL(C_DOUBLE) :: NRIETA(6)
      END TYPE
C     synthetic inflow velocity: RXLPRM(2), RXLPRM(4), LNX..NFZ, ITIME
      TYPE, BIND(C) :: SENGA_SYNTH_INFLOW
        REAL(C_DOUBLE) :: URMS, COFLOW
        INTEGER(C_INT) :: LNX, LNY, LNZ
        INTEGER(C_INT) :: NFY, NFZ
        INTEGER(C_INT) :: ITIME
      END TYPE
      INTERFACE
        INTEGER(C_INT) FUNCTION SENGA_CHEM_LOAD(PATH, CHEM)
     +      BIND(C, NAME='senga_chem_load')
          IMPORT :: C_INT, C_CHAR, SENGA_CHEM
          CHARACTER(KIND=C_CHAR) :: PATH(*)
          TYPE(SENGA_CHEM) :: CHEM
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_DIFF_LOAD(PATH, CHEM, DIFF)
     +      BIND(C, NAME='senga_diff_load')
          IMPORT :: C_INT, C_CHAR, SENGA_CHEM, SENGA_DIFF
          CHARACTER(KIND=C_CHAR) :: PATH(*)
          TYPE(SENGA_CHEM) :: CHEM
          TYPE(SENGA_DIFF) :: DIFF
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_CTX_CREATE(CFG, CHEM, DIFF, CTX)
     +      BIND(C, NAME='senga_ctx_create')
          IMPORT :: C_INT, C_PTR, SENGA_CONFIG, SENGA_CHEM, SENGA_DIFF
          TYPE(SENGA_CONFIG) :: CFG
          TYPE(SENGA_CHEM) :: CHEM
          TYPE(SENGA_DIFF) :: DIFF
          TYPE(C_PTR) :: CTX
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_CTX_DESTROY(CTX)
     +      BIND(C, NAME='senga_ctx_destroy')
          IMPORT :: C_INT, C_PTR
          TYPE(C_PTR), VALUE :: CTX
        END FUNCTION
        TYPE(C_PTR) FUNCTION SENGA_LAST_ERROR()
     +      BIND(C, NAME='senga_last_error')
          IMPORT :: C_PTR
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_UPLOAD_STATE_HOST(CTX, FLDS, TRUN,
     +      ITNDEX) BIND(C, NAME='senga_upload_state_host')
          IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
          TYPE(C_PTR), VALUE :: CTX
          REAL(C_DOUBLE) :: FLDS(*), TRUN(*)
          INTEGER(C_INT32_T) :: ITNDEX(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_DOWNLOAD_STATE_HOST(CTX, FLDS,
     +      TRUN, ITNDEX) BIND(C, NAME='senga_download_state_host')
          IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
          TYPE(C_PTR), VALUE :: CTX
          REAL(C_DOUBLE) :: FLDS(*), TRUN(*)
          INTEGER(C_INT32_T) :: ITNDEX(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_SUBSTAGE(CTX, IRKSTP)
     +      BIND(C, NAME='senga_substage')
          IMPORT :: C_INT, C_PTR
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: IRKSTP
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_STEP_GRAPH(CTX, NSTEPS)
     +      BIND(C, NAME='senga_step_graph')
          IMPORT :: C_INT, C_PTR
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: NSTEPS
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_GET_STATUS(CTX, ISTAT)
     +      BIND(C, NAME='senga_get_status')
          IMPORT :: C_INT, C_PTR
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT) :: ISTAT
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_GET_TSTEP(CTX, TSTEP, ERRMAX,
     +      INDERR) BIND(C, NAME='senga_get_tstep')
          IMPORT :: C_INT, C_PTR, C_DOUBLE
          TYPE(C_PTR), VALUE :: CTX
          REAL(C_DOUBLE) :: TSTEP, ERRMAX
          INTEGER(C_INT) :: INDERR
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_SET_NSCBC(CTX, BC)
     +      BIND(C, NAME='senga_set_nscbc')
          IMPORT :: C_INT, C_PTR, SENGA_NSCBC
          TYPE(C_PTR), VALUE :: CTX
          TYPE(SENGA_NSCBC) :: BC
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_SET_SYNTHETIC_INFLOW(CTX, P)
     +      BIND(C, NAME='senga_set_synthetic_inflow')
          IMPORT :: C_INT, C_PTR, SENGA_SYNTH_INFLOW
          TYPE(C_PTR), VALUE :: CTX
          TYPE(SENGA_SYNTH_INFLOW) :: P
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_SET_TRANSPORT(CTX, MIXW, MIXP,
     +      SORET, DUFOUR, WMLTDR) BIND(C, NAME='senga_set_transport')
          IMPORT :: C_INT, C_PTR, C_DOUBLE
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: MIXW, MIXP, SORET, DUFOUR
          REAL(C_DOUBLE), VALUE :: WMLTDR
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_SET_RADIATION(CTX, RADN)
     +      BIND(C, NAME='senga_set_radiation')
          IMPORT :: C_INT, C_PTR, SENGA_RADN
          TYPE(C_PTR), VALUE :: CTX
          TYPE(SENGA_RADN) :: RADN
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_FILTER(CTX, MODE)
     +      BIND(C, NAME='senga_filter')
          IMPORT :: C_INT, C_PTR
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: MODE
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_TEMPIN_HOST(CTX, TRIN, TRUN,
     +      ITNDEX, PRUN) BIND(C, NAME='senga_tempin_host')
          IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
          TYPE(C_PTR), VALUE :: CTX
          REAL(C_DOUBLE), VALUE :: TRIN
          REAL(C_DOUBLE) :: TRUN(*), PRUN(*)
          INTEGER(C_INT32_T) :: ITNDEX(*)
        END FUNCTION
C       DFBYDX..D2FDYZ on the reference's own arrays: FUNCTN is the
C       halo-extended (1-NHALO:N+NHALO per direction, NHALO = 5) array,
C       FDERIV the interior result (src/dfbydx.f:36-37).
        INTEGER(C_INT) FUNCTION SENGA_DERIV_BIG_HOST(CTX, KIND, FUNCTN,
     +      FDERIV) BIND(C, NAME='senga_deriv_big_host')
          IMPORT :: C_INT, C_PTR, C_DOUBLE
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: KIND
          REAL(C_DOUBLE) :: FUNCTN(*), FDERIV(*)
        END FUNCTION
        INTEGER(C_INT) FUNCTION SENGA_DERIV_HOST(CTX, KIND, F, D)
     +      BIND(C, NAME='senga_deriv_host')
          IMPORT :: C_INT, C_PTR, C_DOUBLE
          TYPE(C_PTR), VALUE :: CTX
          INTEGER(C_INT), VALUE :: KIND
          REAL(C_DOUBLE) :: F(*), D(*)
        END FUNCTION
      END INTERFACE
C     the device context of this rank's box (created once after INDATA)
      TYPE(C_PTR), SAVE :: GPUCTX = C_NULL_PTR
      END MODULE SENGA_GPU
