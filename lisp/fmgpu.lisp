;;; -*- mode: lisp; -*-
;;;
;;; fmgpu.lisp -- Femlisp binding of libfmgpu.so (the B200 multigrid solve
;;; path).  Written for Femlisp's fl.port foreign-function layer
;;; (src/basic/port.lisp:360-547) in the style of src/alien/superlu.lisp:57-75.
;;;
;;; Not exercised here: no Common Lisp implementation is available where this
;;; library is built and tested.  The C side is tested through the same C-ABI
;;; from Python (tests/).
;;;
;;; Load with (fl.port:load-foreign-library "libfmgpu.so") after adding the
;;; library path to fl.start's foreign-library configuration
;;; (src/config/femlisp-config.lisp:65-93).

(defpackage "FL.FMGPU"
  (:use "COMMON-LISP" "FL.MATLISP" "FL.ITERATION")
  (:export "<GPU-LINEAR-SOLVER>" "GPU-SOLVE" "GPU-CONTEXT"))

(in-package "FL.FMGPU")

;;;; constants of include/fmgpu.h

(defconstant +fmg-ok+ 0)
(defconstant +fmg-k-const+ 0)
(defconstant +fmg-k-cell+ 1)
(defconstant +fmg-f-const+ 2)
(defconstant +fmg-f-ip+ 3)
(defconstant +fmg-jacobi+ 0)
(defconstant +fmg-sor+ 1)
(defconstant +fmg-ssc+ 2)
(defconstant +fmg-psc+ 3)
(defconstant +fmg-method-mg+ 0)
(defconstant +fmg-method-cg-mg+ 1)
(defconstant +fmg-multiplicative+ 0)
(defconstant +fmg-additive+ 1)
(defconstant +fmg-csr+ 0)
(defconstant +fmg-ccs+ 1)

;;;; foreign functions (handles are passed as (* :char) pointers)

(fl.port:def-function ("fmg_init" fmg-init)
    ((device :int) (ctx (* (* :char))))
  :returning :int)

(fl.port:def-function ("fmg_finalize" fmg-finalize)
    ((ctx (* :char)))
  :returning :int)

(fl.port:def-function ("fmg_grid_create" fmg-grid-create)
    ((ctx (* :char)) (dim :int) (order :int) (ncomp :int) (n0 :int)
     (top-level :int) (base-level :int) (dirichlet-mask :int)
     (grid (* (* :char))))
  :returning :int)

(fl.port:def-function ("fmg_set_coefficient" fmg-set-coefficient)
    ((grid (* :char)) (kind :int) (values (* :double)) (n :long))
  :returning :int)

(fl.port:def-function ("fmg_assemble" fmg-assemble)
    ((grid (* :char)))
  :returning :int)

(fl.port:def-function ("fmg_vec_create" fmg-vec-create)
    ((grid (* :char)) (level :int) (vec (* (* :char))))
  :returning :int)

(fl.port:def-function ("fmg_vec_get" fmg-vec-get)
    ((vec (* :char)) (host (* :double)) (n :long))
  :returning :int)

;;; fmg_solve takes a pointer to an fmg_solve_cfg struct; it is passed as a
;;; byte vector laid out like the C struct (see %cfg-bytes).
(fl.port:def-function ("fmg_solve" fmg-solve)
    ((grid (* :char)) (cfg (* :char)) (x (* :char))
     (hist (* :double)) (hist-len :int) (nsteps (* :int)) (status (* :int)))
  :returning :int)

(fl.port:def-function ("fmg_set_matrix" fmg-set-matrix)
    ((grid (* :char)) (level :int) (layout :int) (starts (* :int)) (indices (* :int))
     (values (* :double)) (n :long))
  :returning :int)

(fl.port:def-function ("fmg_grid_create_algebraic" fmg-grid-create-algebraic)
    ((ctx (* :char)) (nlevels :int) (sizes (* :long)) (grid (* (* :char))))
  :returning :int)

(fl.port:def-function ("fmg_set_interpolation" fmg-set-interpolation)
    ((grid (* :char)) (fine-level :int) (layout :int) (starts (* :int)) (indices (* :int))
     (values (* :double)) (nfine :long) (ncoarse :long))
  :returning :int)

(fl.port:def-function ("fmg_set_rhs" fmg-set-rhs)
    ((grid (* :char)) (values (* :double)) (n :long))
  :returning :int)

(fl.port:def-function ("fmg_grid_destroy" fmg-grid-destroy)
    ((grid (* :char)))
  :returning :int)

(fl.port:def-function ("fmg_last_error" fmg-last-error)
    ((ctx (* :char)) (buf (* :char)) (len :int))
  :returning :int)

(fl.port:def-function ("fmg_vec_set" fmg-vec-set)
    ((vec (* :char)) (host (* :double)) (n :long))
  :returning :int)

(fl.port:def-function ("fmg_vec_destroy" fmg-vec-destroy)
    ((vec (* :char)))
  :returning :int)

;;; one application of the <geometric-cs> iterator (b and r may be the same
;;; vector: the alias inside <cg>)
(fl.port:def-function ("fmg_vcycle" fmg-vcycle)
    ((grid (* :char)) (cfg (* :char)) (x (* :char)) (b (* :char)) (r (* :char)))
  :returning :int)

;;; the mixed-precision solve and the learned damping
(fl.port:def-function ("fmg_solve_mixed" fmg-solve-mixed)
    ((grid (* :char)) (cfg (* :char)) (mcfg (* :char)) (x (* :char)) (hist (* :double))
     (hist-len :int) (nouter (* :int)) (ninner (* :int)) (status (* :int)))
  :returning :int)

(fl.port:def-function ("fmg_net_load" fmg-net-load)
    ((ctx (* :char)) (path :c-string) (out (* (* :char))))
  :returning :int)

(fl.port:def-function ("fmg_net_destroy" fmg-net-destroy)
    ((net (* :char)))
  :returning :int)

(fl.port:def-function ("fmg_net_apply" fmg-net-apply)
    ((net (* :char)) (grid (* :char)))
  :returning :int)

(fl.port:def-function ("fmg_learned_judge_mixed" fmg-learned-judge-mixed)
    ((grid (* :char)) (cfg (* :char)) (mcfg (* :char)) (rho-plain (* :double))
     (rho-learned (* :double)) (accepted (* :int)))
  :returning :int)

(defun check (status what)
  (unless (= status +fmg-ok+)
    (error "libfmgpu: ~A failed with status ~D" what status)))

;;;; a solver class usable on a Femlisp blackboard

(defclass <gpu-linear-solver> (<linear-solver>)
  ((smoother :initarg :smoother :initform :jacobi)
   (damp :initarg :damp :initform 0.6d0)
   (pre-steps :initarg :pre-steps :initform 1)
   (post-steps :initarg :post-steps :initform 1)
   (base-level :initarg :base-level :initform 0)
   (reduction :initarg :reduction :initform 1d-10)
   (maxsteps :initarg :maxsteps :initform 200))
  (:documentation "<cg> preconditioned by <geometric-cs>, run by libfmgpu on
the GPU; SMOOTHER is :jacobi, :sor, :ssc or :psc (the vertex-centred
geometric-ssc / geometric-psc, the default of higher-order discretisations).  The problem must be a cdr problem on a uniformly refined unit
n-cube with Lagrange Q1/Q2; the coefficients are sampled on the host."))

(defvar *gpu-context* nil)

(defun gpu-context ()
  (or *gpu-context*
      (let ((ctx (make-array 1 :element-type '(unsigned-byte 64))))
        (check (fl.port:foreign-call #'fmg-init 0 ctx) "fmg_init")
        (setq *gpu-context* (aref ctx 0)))))

(defun %cfg-bytes (method smoother damp pre post rtol maxsteps)
  "fmg_solve_cfg laid out as the C struct (72 bytes with x86-64 alignment;
the last int, fmg at byte 64, stays 0: V/W cycles)."
  (let ((v (make-array 72 :element-type '(unsigned-byte 8) :initial-element 0)))
    (flet ((int! (off x) (setf (fl.port:sap-ref-32 v off) x))
           (dbl! (off x) (setf (fl.port:sap-ref-double v off) x)))
      (int! 0 method) (int! 4 smoother) (dbl! 8 damp)
      (int! 16 pre) (int! 20 post) (int! 24 1) (int! 28 0)
      (dbl! 32 1d0) (dbl! 40 rtol) (dbl! 48 0d0) (int! 56 maxsteps)
      (int! 60 +fmg-multiplicative+))
    v))

(defun gpu-solve (solver dim order level kcell &key (source 1d0))
  "Assemble and solve on the GPU; returns the nodal solution (lexicographic,
x fastest) and the :defnorm history."
  (with-slots (smoother damp pre-steps post-steps base-level reduction maxsteps) solver
    (let ((grid (make-array 1 :element-type '(unsigned-byte 64)))
          (x (make-array 1 :element-type '(unsigned-byte 64)))
          (hist (make-array (+ maxsteps 2) :element-type 'double-float))
          (nsteps (make-array 1 :element-type '(signed-byte 32)))
          (status (make-array 1 :element-type '(signed-byte 32))))
      (check (fl.port:foreign-call #'fmg-grid-create (gpu-context) dim order 1 1 level
                                   base-level (1- (expt 2 (* 2 dim))) grid)
             "fmg_grid_create")
      (if kcell
          (check (fl.port:foreign-call #'fmg-set-coefficient (aref grid 0) +fmg-k-cell+
                                       kcell (length kcell))
                 "fmg_set_coefficient")
          nil)
      (let ((f (make-array 1 :element-type 'double-float :initial-element source)))
        (check (fl.port:foreign-call #'fmg-set-coefficient (aref grid 0) +fmg-f-const+ f 1)
               "fmg_set_coefficient"))
      (check (fl.port:foreign-call #'fmg-assemble (aref grid 0)) "fmg_assemble")
      (check (fl.port:foreign-call #'fmg-vec-create (aref grid 0) level x) "fmg_vec_create")
      (check (fl.port:foreign-call
              #'fmg-solve (aref grid 0)
              (%cfg-bytes +fmg-method-cg-mg+
                          (ecase smoother
                            (:jacobi +fmg-jacobi+) (:sor +fmg-sor+)
                            (:ssc +fmg-ssc+) (:psc +fmg-psc+))   ; geometric-ssc / -psc
                          damp pre-steps post-steps reduction maxsteps)
              (aref x 0) hist (length hist) nsteps status)
             "fmg_solve")
      (let* ((n (expt (1+ (* order (expt 2 level))) dim))
             (sol (make-array n :element-type 'double-float)))
        (check (fl.port:foreign-call #'fmg-vec-get (aref x 0) sol n) "fmg_vec_get")
        (values sol (subseq hist 0 (1+ (aref nsteps 0))))))))

;;;; matrices Femlisp assembled itself

(defun lexicographic-keys (matrix)
  "The row keys of MATRIX in the library's node order: by the midpoint of the
key's cell, last coordinate slowest (the numbering of sparse-matrix->ccs is
the order of the keys it is given, sparselu.lisp:226-233)."
  (let ((keys (coerce (fl.matlisp:row-keys matrix) 'vector)))
    (flet ((mid (key) (fl.mesh:midpoint (fl.mesh:representative key))))
      (sort keys (lambda (a b)
                   (let ((pa (mid a)) (pb (mid b)))
                     (loop for k from (1- (length pa)) downto 0
                           when (< (aref pa k) (aref pb k)) return t
                           when (> (aref pa k) (aref pb k)) return nil
                           finally (return nil))))))))

(defun upload-level-matrix (grid level matrix)
  "Hands the level matrix MATRIX (a <sparse-matrix> of the structured
hierarchy, constraints eliminated) to the library through fmg_set_matrix in
the compressed-column form of sparse-matrix->ccs."
  (let* ((keys (lexicographic-keys matrix))
         (ccs (fl.matlisp:sparse-matrix->ccs matrix :keys keys))
         (pattern (fl.matlisp:pattern ccs))
         (starts (slot-value pattern 'fl.matlisp::starts))
         (indices (slot-value pattern 'fl.matlisp::indices))
         (n (1- (length starts))))
    (check (fl.port:foreign-call #'fmg-set-matrix grid level +fmg-ccs+ starts indices
                                 (fl.matlisp:store ccs) n)
           "fmg_set_matrix")))

;;;; hierarchies on unstructured or adaptively refined meshes

(defun upload-algebraic-hierarchy (matrices interpolations rhs)
  "MATRICES: the level matrices of a multilevel decomposition, coarsest
first (<sparse-matrix>, constraints eliminated, multilevel-decomposition
geomg.lisp:109-142); INTERPOLATIONS: the constrained interpolation into each
level above the coarsest (constrained-interpolation-matrix,
constraints.lisp:58-72), coarsest first; RHS: the top-level right-hand side
as a double vector in the top level's key order.  Returns the grid handle."
  (let* ((keys (mapcar (lambda (m) (coerce (fl.matlisp:row-keys m) 'vector)) matrices))
         (sizes (map '(vector (signed-byte 64)) #'length keys))
         (grid (make-array 1 :element-type '(unsigned-byte 64))))
    (check (fl.port:foreign-call #'fmg-grid-create-algebraic (gpu-context) (length sizes) sizes grid)
           "fmg_grid_create_algebraic")
    (loop for m in matrices for k in keys for level from 0 do
      (let* ((ccs (fl.matlisp:sparse-matrix->ccs m :keys k))
             (pattern (fl.matlisp:pattern ccs)))
        (check (fl.port:foreign-call #'fmg-set-matrix (aref grid 0) level +fmg-ccs+
                                     (slot-value pattern 'fl.matlisp::starts)
                                     (slot-value pattern 'fl.matlisp::indices)
                                     (fl.matlisp:store ccs) (length k))
               "fmg_set_matrix")))
    (loop for i in interpolations for level from 1 do
      (let* ((ccs (fl.matlisp:sparse-matrix->ccs i :row-keys (nth level keys) :col-keys (nth (1- level) keys)))
             (pattern (fl.matlisp:pattern ccs)))
        (check (fl.port:foreign-call #'fmg-set-interpolation (aref grid 0) level +fmg-ccs+
                                     (slot-value pattern 'fl.matlisp::starts)
                                     (slot-value pattern 'fl.matlisp::indices)
                                     (fl.matlisp:store ccs) (length (nth level keys))
                                     (length (nth (1- level) keys)))
               "fmg_set_interpolation")))
    (check (fl.port:foreign-call #'fmg-set-rhs (aref grid 0) rhs (length rhs)) "fmg_set_rhs")
    (aref grid 0)))

;;;; the mixed-precision solve with the learned damping

(defun %mixed-cfg-bytes (inner-rtol max-inner max-outer matrix-free)
  "fmg_mixed_cfg laid out as the C struct (24 bytes)."
  (let ((v (make-array 24 :element-type '(unsigned-byte 8) :initial-element 0)))
    (setf (fl.port:sap-ref-double v 0) inner-rtol
          (fl.port:sap-ref-32 v 8) max-inner
          (fl.port:sap-ref-32 v 12) max-outer
          (fl.port:sap-ref-32 v 16) (if matrix-free 1 0))
    v))

(defun gpu-solve-mixed (grid level weights-path &key (damp 0.6d0) (reduction 1d-10) (maxsteps 200))
  "On an assembled GRID whose top level is LEVEL: installs the per-node damping the network in
WEIGHTS-PATH predicts, lets the plain cycle judge it (it stays only if no
worse), and solves with FP64 flexible CG around the FP32/BF16 V(1,1) Jacobi
cycle.  Returns the solution vector handle and the :defnorm history."
  (let* ((ctx (gpu-context))
         (net (make-array 1 :element-type '(unsigned-byte 64)))
         (x (make-array 1 :element-type '(unsigned-byte 64)))
         (cfg (%cfg-bytes +fmg-method-cg-mg+ +fmg-jacobi+ damp 1 1 reduction maxsteps))
         (mcfg (%mixed-cfg-bytes 1d-5 200 20 t))
         (rho-plain (make-array 1 :element-type 'double-float))
         (rho-learned (make-array 1 :element-type 'double-float))
         (accepted (make-array 1 :element-type '(signed-byte 32)))
         (hist (make-array (+ maxsteps 24) :element-type 'double-float))
         (nouter (make-array 1 :element-type '(signed-byte 32)))
         (ninner (make-array 1 :element-type '(signed-byte 32)))
         (status (make-array 1 :element-type '(signed-byte 32))))
    (check (fl.port:foreign-call #'fmg-net-load ctx weights-path net) "fmg_net_load")
    (unwind-protect
         (progn
           (check (fl.port:foreign-call #'fmg-net-apply (aref net 0) grid) "fmg_net_apply")
           (check (fl.port:foreign-call #'fmg-learned-judge-mixed grid cfg mcfg rho-plain rho-learned accepted)
                  "fmg_learned_judge_mixed"))
      (fl.port:foreign-call #'fmg-net-destroy (aref net 0)))
    (check (fl.port:foreign-call #'fmg-vec-create grid level x) "fmg_vec_create")
    (check (fl.port:foreign-call #'fmg-solve-mixed grid cfg mcfg (aref x 0) hist (length hist)
                                 nouter ninner status)
           "fmg_solve_mixed")
    (values (aref x 0) (subseq hist 0 (+ (aref nouter 0) (aref ninner 0) 1)))))
