# One configuration of HiRep's library and the hr_ref server (called by Makefile
# with REF, OUT, CFG, NG, REPR and MACRO set).
GAUGE := GAUGE_SUN
B     := $(OUT)/_build/$(CFG)
GEN   := $(B)/gen
EXE   := $(OUT)/$(CFG)/hr_ref

EXCL := Geometry/blocked.c Inverters/HBiCGstab.c Inverters/BiCGstab_mshift.c \
        Inverters/HBiCGstab_mshift.c Inverters/dirac_eva.c Observables/trunc_hairpin.c
ifneq ($(NG),2)
EXCL += Utils/HYP_smearing.c
endif

SRCS := $(filter-out $(addprefix $(REF)/LibHR/,$(EXCL)),$(sort $(wildcard $(REF)/LibHR/*/*.c)))
OBJS := $(patsubst $(REF)/LibHR/%.c,$(B)/obj/%.o,$(SRCS)) $(B)/obj/Utils/suN_exp.o

# the macros of HiRep's MkFlags for a serial even-odd build with the
# configurations' boundary conditions (antiperiodic in time)
CPP := -D$(REPR) -DREPR_NAME=\"$(REPR)\" -D$(GAUGE) -DBC_T_ANTIPERIODIC -DBC_X_PERIODIC \
       -DBC_Y_PERIODIC -DBC_Z_PERIODIC -DUPDATE_EO -DNDEBUG -DCHECK_SPINOR_MATCHING -DIO_FLUSH $(MACRO)
INC := -I$(GEN) -I$(REF)/Include
CFLAGS := -std=gnu99 -O3 -fopenmp -w

HDRS := $(GEN)/suN.h $(GEN)/suN_types.h $(GEN)/suN_repr_func.h $(GEN)/cinfo.c $(GEN)/approx_data.db

all: $(EXE)

$(EXE): hr_ref.c $(B)/libhr.a
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) hr_ref.c -o $@ $(B)/libhr.a -lm

$(B)/libhr.a: $(OBJS)
	@rm -f $@
	ar rcs $@ $(OBJS)

$(B)/obj/%.o: $(REF)/LibHR/%.c $(HDRS)
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) -c $< -o $@

$(B)/obj/Utils/suN_exp.o: $(GEN)/suN_exp.c $(HDRS)
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) -I$(REF)/LibHR/Utils -c $< -o $@

# write_suN_headers.pl NG REPR WITH_QUATERNIONS GAUGE_GROUP writes both headers into its cwd
$(GEN)/suN.h $(GEN)/suN_types.h &:
	@mkdir -p $(GEN)
	cd $(GEN) && perl $(REF)/Make/Utils/write_suN_headers.pl $(NG) $(REPR) 0 $(GAUGE) > /dev/null

$(GEN)/writeREPR: $(REF)/Make/Utils/autosun/main.cc
	@mkdir -p $(GEN)
	g++ -O2 $< -o $@ -D_$(REPR)_ -D_$(GAUGE)_ -D_PICA_STYLE_ -DNDEBUG

$(GEN)/suN_repr_func.h: $(GEN)/writeREPR
	$(GEN)/writeREPR $(NG) $(REF)/Include/TMPL/suN_repr_func.h.tmpl > $@

$(GEN)/suN_exp.c: $(GEN)/writeREPR
	$(GEN)/writeREPR $(NG) $(REF)/LibHR/Utils/TMPL/suN_exp.c.tmpl > $@

$(GEN)/cinfo.c:
	@mkdir -p $(GEN)
	cd $(GEN) && rm -f cinfo.lock && bash $(REF)/Make/Utils/cinfo.sh $(REF)/Make $(REF) $(CPP) > /dev/null 2>&1; test -s cinfo.c

$(GEN)/approx_data.db:
	@mkdir -p $(GEN)
	cd $(REF)/LibHR/Update/remez && cat approx_* | perl ./mkappdata.pl > $@

.PHONY: all

# ---------------------------------------------------------------------------
# HiRep's own check programs linked through the drop-in binding
# (hirep_b200/shim/hrgpu_hirep.c) to the GPU library: the replaced functions
# are redirected with the linker's --wrap, HiRep's sources stay as they are.
# Needs hirep_b200/libhrgpu.so built first.
SHIM     := $(abspath ../../hirep_b200/shim/hrgpu_hirep.c)
GPULIB   := $(abspath ../../hirep_b200)
CUDA     ?= /usr/local/cuda
CHECKS   := DiracOperator/check_diracoperator_1 DiracOperator/check_diracoperator_3 \
            DiracOperator/check_diracoperator_6 Inverters/check_inverters_1 Inverters/check_inverters_6
WRAPPED  := represent_gauge_field compute_clover_term set_dirac_mass getMVM Dphi_ Dphi g5Dphi g5Dphi_sq \
            Dphi_eopre Dphi_oepre g5Dphi_eopre g5Dphi_eopre_sq Dphi_flt_ Dphi_flt g5Dphi_flt g5Dphi_sq_flt \
            Dphi_eopre_flt g5Dphi_eopre_flt g5Dphi_eopre_sq_flt Cphi g5Cphi g5Cphi_sq Cphi_eopre g5Cphi_eopre \
            g5Cphi_eopre_sq Cphi_diag Cphi_diag_inv cg_mshift fermion_force_begin force_fermion_core fermion_force_end
SHIMEXE  := $(foreach c,$(CHECKS),$(OUT)/$(CFG)/shim/$(notdir $(c)))

shim: $(SHIMEXE)

$(B)/shim/hrgpu_hirep.o: $(SHIM) $(HDRS) ../../include/hrgpu.h
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) -I../../include -I$(CUDA)/include -c $< -o $@

$(B)/shim/%.o: $(REF)/TestProgram/DiracOperator/%.c $(HDRS)
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) -c $< -o $@

$(B)/shim/%.o: $(REF)/TestProgram/Inverters/%.c $(HDRS)
	@mkdir -p $(dir $@)
	gcc $(CFLAGS) $(CPP) $(INC) -c $< -o $@

$(OUT)/$(CFG)/shim/%: $(B)/shim/%.o $(B)/shim/hrgpu_hirep.o $(B)/libhr.a $(GPULIB)/libhrgpu.so
	@mkdir -p $(dir $@)
	gcc -fopenmp -o $@ $< $(B)/shim/hrgpu_hirep.o $(B)/libhr.a $(addprefix -Wl$(comma)--wrap=,$(WRAPPED)) \
	    -L$(GPULIB) -lhrgpu -L$(CUDA)/lib64 -lcudart -lm \
	    -Wl,-rpath,'$$ORIGIN/../../../../hirep_b200' -Wl,-rpath,$(CUDA)/lib64

comma := ,
.PHONY: shim
