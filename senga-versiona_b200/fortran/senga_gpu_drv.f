C     Thin glue between SENGA2's COMMON blocks and the device path, for a
C     serial (one-rank, one-GPU) run: compiled with the reference's own
C     sources and its com_senga2.h, it replaces the per-substage sequence
C     of src/senga2.f:113-159 by one call per RK step. The reference's
C     routines keep everything else (input, output, statistics).
C
C       after INDATA (src/indata.f:1589):   CALL GPUINI
C       the RK loop body (src/senga2.f:113-159, five substages):
C                                           CALL GPUSTP
C       before a dump/report (src/output.f:241,273) and FINISH:
C                                           CALL GPUGET
C
C     Interior (std) ranges only cross the boundary; the conserved fields
C     are packed field-slowest (rho, rho u, rho v, rho w, rho E, rho Y_k),
C     as include/senga_gpu.h states. ITNDEX crosses as its first
C     1 + (NSPEC-1)/NSPIMX words, each carrying the intervals of NSPIMX =
C     15 species in base NTBASE = 4 (src/temper.f:195-201), the packing of
C     the device's index.

      SUBROUTINE GPUINI
      USE ISO_C_BINDING
      USE SENGA_GPU
      INCLUDE 'com_senga2.h'
      TYPE(SENGA_CONFIG) CFG
      TYPE(SENGA_CHEM), SAVE :: GCHEM
      TYPE(SENGA_DIFF), SAVE :: GDIFF
      INTEGER ISTAT
      CFG%NX = NXNODE
      CFG%NY = NYNODE
      CFG%NZ = NZNODE
      CFG%XGDLEN = XGDLEN
      CFG%YGDLEN = YGDLEN
      CFG%ZGDLEN = ZGDLEN
      CFG%NEND(1) = NENDXL
      CFG%NEND(2) = NENDXR
      CFG%NEND(3) = NENDYL
      CFG%NEND(4) = NENDYR
      CFG%NEND(5) = NENDZL
      CFG%NEND(6) = NENDZR
      CFG%TSTEP = TSTEP
      CFG%ADAPTIVE = NSTPSW
      CFG%DEVICE = 0
      ISTAT = SENGA_CHEM_LOAD('chem.dat'//C_NULL_CHAR, GCHEM)
      IF(ISTAT.NE.0)CALL GPUERR('senga_chem_load', ISTAT)
      IF(FLMAVT)THEN
        ISTAT = SENGA_DIFF_LOAD('diff.dat'//C_NULL_CHAR, GCHEM, GDIFF)
      ELSE
        ISTAT = SENGA_DIFF_LOAD(C_NULL_CHAR, GCHEM, GDIFF)
      ENDIF
      IF(ISTAT.NE.0)CALL GPUERR('senga_diff_load', ISTAT)
      ISTAT = SENGA_CTX_CREATE(CFG, GCHEM, GDIFF, GPUCTX)
      IF(ISTAT.NE.0)CALL GPUERR('senga_ctx_create', ISTAT)
      CALL GPUPUT
      RETURN
      END

      SUBROUTINE GPUPUT
C     COMMON registers -> device (both RK registers = xRUN)
      USE ISO_C_BINDING
      USE SENGA_GPU
      INCLUDE 'com_senga2.h'
      DOUBLE PRECISION, ALLOCATABLE :: FLDS(:,:,:,:), TSTD(:,:,:)
      INTEGER(C_INT32_T), ALLOCATABLE :: ISTD(:,:,:,:)
      INTEGER IC,JC,KC,ISPEC,ISTAT,IW,NWORD
      NWORD = 1 + (NSPEC-1)/NSPIMX
      ALLOCATE(FLDS(NXNODE,NYNODE,NZNODE,5+NSPEC))
      ALLOCATE(TSTD(NXNODE,NYNODE,NZNODE))
      ALLOCATE(ISTD(NXNODE,NYNODE,NZNODE,NWORD))
      DO KC = 1,NZNODE
        DO JC = 1,NYNODE
          DO IC = 1,NXNODE
            FLDS(IC,JC,KC,1) = DRUN(IC,JC,KC)
            FLDS(IC,JC,KC,2) = URUN(IC,JC,KC)
            FLDS(IC,JC,KC,3) = VRUN(IC,JC,KC)
            FLDS(IC,JC,KC,4) = WRUN(IC,JC,KC)
            FLDS(IC,JC,KC,5) = ERUN(IC,JC,KC)
            DO ISPEC = 1,NSPEC
              FLDS(IC,JC,KC,5+ISPEC) = YRUN(IC,JC,KC,ISPEC)
            ENDDO
            TSTD(IC,JC,KC) = TRUN(IC,JC,KC)
            DO IW = 1,NWORD
              ISTD(IC,JC,KC,IW) = ITNDEX(IC,JC,KC,IW)
            ENDDO
          ENDDO
        ENDDO
      ENDDO
      ISTAT = SENGA_UPLOAD_STATE_HOST(GPUCTX, FLDS, TSTD, ISTD)
      IF(ISTAT.NE.0)CALL GPUERR('senga_upload_state_host', ISTAT)
      DEALLOCATE(FLDS, TSTD, ISTD)
      RETURN
      END

      SUBROUTINE GPUSTP
C     one RK step (five substages, BOUNTT, ADAPTT when NSTPSW = 1) on the
C     device; STOP where the reference's TEMPER would (src/temper.f:156)
      USE ISO_C_BINDING
      USE SENGA_GPU
      INCLUDE 'com_senga2.h'
      INTEGER ISTAT, IFLAG, INDERR
      DOUBLE PRECISION ERRMAX
      ISTAT = SENGA_STEP_GRAPH(GPUCTX, 1)
      IF(ISTAT.NE.0)CALL GPUERR('senga_step_graph', ISTAT)
      ISTAT = SENGA_GET_STATUS(GPUCTX, IFLAG)
      IF(ISTAT.NE.0)CALL GPUERR('senga_get_status', ISTAT)
      IF(MOD(IFLAG,2).EQ.1)THEN
        WRITE(6,*)'Fatal: TEMPER: no convergence on the device'
        STOP
      ENDIF
      IF(NSTPSW.EQ.1)THEN
        ISTAT = SENGA_GET_TSTEP(GPUCTX, TSTEP, ERRMAX, INDERR)
        IF(ISTAT.NE.0)CALL GPUERR('senga_get_tstep', ISTAT)
      ENDIF
      RETURN
      END

      SUBROUTINE GPUGET
C     device -> COMMON registers (xRUN, and xRHS = xRUN as after FINCOM)
      USE ISO_C_BINDING
      USE SENGA_GPU
      INCLUDE 'com_senga2.h'
      DOUBLE PRECISION, ALLOCATABLE :: FLDS(:,:,:,:), TSTD(:,:,:)
      INTEGER(C_INT32_T), ALLOCATABLE :: ISTD(:,:,:,:)
      INTEGER IC,JC,KC,ISPEC,ISTAT,IW,NWORD
      NWORD = 1 + (NSPEC-1)/NSPIMX
      ALLOCATE(FLDS(NXNODE,NYNODE,NZNODE,5+NSPEC))
      ALLOCATE(TSTD(NXNODE,NYNODE,NZNODE))
      ALLOCATE(ISTD(NXNODE,NYNODE,NZNODE,NWORD))
      ISTAT = SENGA_DOWNLOAD_STATE_HOST(GPUCTX, FLDS, TSTD, ISTD)
      IF(ISTAT.NE.0)CALL GPUERR('senga_download_state_host', ISTAT)
      DO KC = 1,NZNODE
        DO JC = 1,NYNODE
          DO IC = 1,NXNODE
            DRUN(IC,JC,KC) = FLDS(IC,JC,KC,1)
            URUN(IC,JC,KC) = FLDS(IC,JC,KC,2)
            VRUN(IC,JC,KC) = FLDS(IC,JC,KC,3)
            WRUN(IC,JC,KC) = FLDS(IC,JC,KC,4)
            ERUN(IC,JC,KC) = FLDS(IC,JC,KC,5)
            DRHS(IC,JC,KC) = FLDS(IC,JC,KC,1)
            URHS(IC,JC,KC) = FLDS(IC,JC,KC,2)
            VRHS(IC,JC,KC) = FLDS(IC,JC,KC,3)
            WRHS(IC,JC,KC) = FLDS(IC,JC,KC,4)
            ERHS(IC,JC,KC) = FLDS(IC,JC,KC,5)
            DO ISPEC = 1,NSPEC
              YRUN(IC,JC,KC,ISPEC) = FLDS(IC,JC,KC,5+ISPEC)
              YRHS(IC,JC,KC,ISPEC) = FLDS(IC,JC,KC,5+ISPEC)
            ENDDO
            TRUN(IC,JC,KC) = TSTD(IC,JC,KC)
            DO IW = 1,NWORD
              ITNDEX(IC,JC,KC,IW) = ISTD(IC,JC,KC,IW)
            ENDDO
          ENDDO
        ENDDO
      ENDDO
      DEALLOCATE(FLDS, TSTD, ISTD)
      RETURN
      END

      SUBROUTINE GPUERR(WHAT, ISTAT)
C     report a failed call with the library's message and stop
      USE ISO_C_BINDING
      USE SENGA_GPU
      CHARACTER*(*) WHAT
      INTEGER ISTAT, I
      CHARACTER(KIND=C_CHAR), POINTER :: MSG(:)
      CALL C_F_POINTER(SENGA_LAST_ERROR(), MSG, [512])
      WRITE(6,'(A,A,I4)')WHAT,': status ',ISTAT
      DO I = 1,512
        IF(MSG(I).EQ.C_NULL_CHAR)GOTO 10
        WRITE(6,'(A)',ADVANCE='NO')MSG(I)
      ENDDO
   10 WRITE(6,*)
      STOP
      END
